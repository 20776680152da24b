-- Single-Plummer dwarf on the Orphan-stream orbit: the set-up of the reference's golden
-- likelihood tests (nbody/tests/orphan_models/model_4.lua and model_5.lua, driven by
-- nbody/tests/RunTestUnits.lua), restated for this repository's golden checks.
-- Arguments: nbody, variant ("4": Hernquist bulge, vhalo 114, r 28.9, v (-179,106,109);
--                             "5": Plummer bulge,   vhalo 73,  r 28.6, v (-156, 79,107);
--                             "triaxial": Hernquist bulge, the triaxial halo of
--                             nbody/tests/orphan_models/model_triaxial.lua, r 29.5,
--                             v (-183,101,107);
--                             "bar": nbody/tests/orphan_models/model_bar.lua -- Hernquist
--                             bulge, lighter disk, orbiting bar, vhalo 74.61, r 28.8,
--                             v (-170,94,108), evolved to the end of the best-likelihood
--                             window with two bar-calibration runs).
-- An optional third argument holds options: "allterms" turns on every comparison of the
-- likelihood (velocity dispersion, line-of-sight velocity, beta average, distance, proper
-- motions); "bestlike" turns on the best-likelihood scan over the last 5% of the steps.
-- The seed comes from the command line (argSeed), as in the reference tests.

arg = {...}

seed = argSeed
nbody = arg[1]
variant = arg[2] or "5"

assert(seed ~= nil, "seed argument missing")
assert(nbody ~= nil, "body count argument missing")

prng = DSFMT.create(seed)

dwarfMass = 16
dwarfRadius = 0.2

local bulgeIsPlummer = (variant == "5")
local triaxial = (variant == "triaxial")
local bar = (variant == "bar")
local options = arg[3] or ""
local allTerms = string.find(options, "allterms") ~= nil
local bestLike = string.find(options, "bestlike") ~= nil
local haloSpeed = bulgeIsPlummer and 73 or 114
local orbitR = bulgeIsPlummer and 28.6 or 28.9
local orbitV = bulgeIsPlummer and { -156, 79, 107 } or { -179, 106, 109 }
if triaxial then
   orbitR = 29.5
   orbitV = { -183, 101, 107 }
elseif bar then
   orbitR = 28.8
   orbitV = { -170, 94, 108 }
end

-- The best-likelihood window: evolve to its end, (2 - start) * 3.945 Gyr, and start the
-- likelihood scan at start / (2 - start) of that (the bar model's window starts at 0.95).
local windowStart = 0.95
local evolveTime = bar and (2.0 - windowStart) * 3.945 or 3.945

function makePotential()
   if bar then
      return Potential.create{
         spherical = Spherical.hernquist{ mass = 1.52954402e5, scale = 0.7 },
         disk      = Disk.miyamotoNagai{ mass = 4.18972480e5, scaleLength = 6.5, scaleHeight = 0.26 },
         disk2     = Disk.orbitingBar{ mass = 2.689340798e4, scaleLength = 5.4,
                                       patternSpeed = 250.61, startAngle = 0.488692 },
         halo      = Halo.logarithmic{ vhalo = 74.61, scaleLength = 12.0, flattenZ = 1.0 }
      }
   end
   local bulge
   if bulgeIsPlummer then
      bulge = Spherical.plummer{ mass = 1.52954402E5, scale = 0.7 }
   else
      bulge = Spherical.hernquist{ mass = 1.52954402E5, scale = 0.7 }
   end
   return Potential.create{
      spherical = bulge,
      disk      = Disk.miyamotoNagai{ mass = 4.45865888E5, scaleLength = 6.5, scaleHeight = 0.26 },
      disk2     = Disk.none{ mass = 3.0e5 },
      halo      = triaxial
                  and Halo.triaxial{ vhalo = 116, scaleLength = 16.3, flattenZ = 1.43,
                                     flattenX = 1.26, flattenY = 1.0, triaxAngle = 96 }
                  or Halo.logarithmic{ vhalo = haloSpeed, scaleLength = 12, flattenZ = 1 }
   }
end

function makeContext()
   if bar then
      return NBodyCtx.create{
         timestep        = calculateTimestep(dwarfMass, dwarfRadius),
         timeEvolve      = evolveTime,
         timeBack        = 3.945,
         eps2            = calculateEps2(nbody, dwarfRadius, 0),
         criterion       = "sw93",
         useQuad         = true,
         theta           = 1.0,
         useBestLike     = true,
         BestLikeStart   = windowStart / (2.0 - windowStart),
         BetaSigma       = 2.5,
         VelSigma        = 2.5,
         DistSigma       = 2.5,
         PMSigma         = 2.5,
         BetaCorrect     = 1.111,
         VelCorrect      = 1.111,
         DistCorrect     = 1.111,
         PMCorrect       = 1.111,
         IterMax         = 6,
         calibrationRuns = 2
      }
   end
   return NBodyCtx.create{
      timestep      = calculateTimestep(dwarfMass, dwarfRadius),
      timeEvolve    = 3.945,
      eps2          = calculateEps2(nbody, dwarfRadius, 1),
      criterion     = "sw93",
      useQuad       = true,
      theta         = 1.0,
      useBestLike   = bestLike,
      BestLikeStart = 0.95,
      BetaSigma     = 2.5,
      VelSigma      = 2.5,
      DistSigma     = 2.5,
      PMSigma       = 2.5,
      BetaCorrect   = 1.111,
      VelCorrect    = 1.111,
      DistCorrect   = 1.111,
      PMCorrect     = 1.111,
      IterMax       = 6,
      useVelDisp    = allTerms,
      useBetaComp   = allTerms,
      useVlos       = allTerms,
      useDist       = allTerms,
      usePropMot    = allTerms
   }
end

function makeBodies(ctx, potential)
   local finalPosition, finalVelocity = reverseOrbit{
      potential = potential,
      position  = lbrToCartesian(ctx, Vector.create(218, 53.5, orbitR)),
      velocity  = Vector.create(orbitV[1], orbitV[2], orbitV[3]),
      tstop     = 4.0,
      dt        = ctx.timestep / 10.0
   }

   return predefinedModels.plummer{
      nbody       = nbody,
      prng        = prng,
      position    = finalPosition,
      velocity    = finalVelocity,
      mass        = dwarfMass,
      scaleRadius = dwarfRadius,
      ignore      = false
   }
end

function makeHistogram()
   return HistogramParams.create{
      phi = 128.79,
      theta = 54.39,
      psi = 90.70,
      lambdaStart = -50,
      lambdaEnd   = 50,
      lambdaBins  = 34,
      betaStart = -15,
      betaEnd   = 15,
      betaBins  = 1
   }
end
