-- The CPU-runnable two-component dwarf: the sample workunit's two-component Plummer dwarf
-- (nbody/sample_workunits/for_developers.lua, ModelComponents = 2) with its potential, its
-- timestep formula and its softening (calculateEps2), placed directly on its present-day
-- orbit point (l = 218, b = 53.5, r = 28.6 kpc; v = (-156, 79, 107)) without a reverse orbit,
-- TreeCode with quadrupoles.  Only the reference's own Lua functions and sampler run here.
-- Arguments (all optional):
--   1 nbody        bodies sampled (default 20000; half of them baryons)
--   2 nbodyEps     the body count calculateEps2 is evaluated at (default: nbody), so that the
--                  softening of a large dwarf can be read without sampling it
--   3 theta        opening angle (default 1.0)
--   4 nsteps       the run's step count: timeEvolve = nsteps * the formula's timestep, which
--                  NBodyCtx.create then corrects as nbCorrectTimestep does (default 200)
-- The seed comes from the command line (argSeed).

arg = {...}

assert(argSeed ~= nil, "seed argument missing")
prng = DSFMT.create(argSeed)

nbody = tonumber(arg[1] or "20000")
nbodyEps = tonumber(arg[2] or arg[1] or "20000")
theta = tonumber(arg[3] or "1.0")
nsteps = tonumber(arg[4] or "200")

-- the sample workunit's dwarf parameters and their derived dark component
local massL, rscaleL = 12.0, 0.2
local radiusRatio, massRatio = 0.2, 0.2
local rscaleD = rscaleL / radiusRatio * (1.0 - radiusRatio)
local massD = massL / massRatio * (1.0 - massRatio)

-- the two-component timestep: the smaller of the two components' enclosed-mass crossing times
local function twoComponentTimestep()
   local encD = massD * rscaleL ^ 3 * (rscaleL ^ 2 + rscaleD ^ 2) ^ (-3.0 / 2.0)
   local encL = massL * rscaleD ^ 3 * (rscaleL ^ 2 + rscaleD ^ 2) ^ (-3.0 / 2.0)
   local sL = rscaleL ^ 3 / (encD + massL)
   local sD = rscaleD ^ 3 / (encL + massD)
   local s = sL
   if sD < sL then s = sD end
   return (1.0 / 100.0) * (pi_4_3 * s) ^ (1.0 / 2.0)
end

local dt = twoComponentTimestep()

function makePotential()
   return Potential.create{
      spherical = Spherical.hernquist{ mass = 1.52954402e5, scale = 0.7 },
      disk      = Disk.miyamotoNagai{ mass = 4.45865888e5, scaleLength = 6.5, scaleHeight = 0.26 },
      disk2     = Disk.none{ mass = 3.0e5 },
      halo      = Halo.logarithmic{ vhalo = 74.61, scaleLength = 12.0, flattenZ = 1.0 }
   }
end

function makeContext()
   return NBodyCtx.create{
      timeEvolve  = nsteps * dt,
      timestep    = dt,
      eps2        = calculateEps2(nbodyEps, rscaleL, rscaleD, massL, massD, 0),
      criterion   = "TreeCode",
      useQuad     = true,
      theta       = theta,
      BetaSigma   = 2.5,
      VelSigma    = 2.5,
      DistSigma   = 2.5,
      PMSigma     = 2.5,
      BetaCorrect = 1.111,
      VelCorrect  = 1.111,
      DistCorrect = 1.111,
      PMCorrect   = 1.111,
      IterMax     = 6
   }
end

function makeBodies(ctx, potential)
   return predefinedModels.mixeddwarf{
      nbody        = nbody,
      nbody_baryon = nbody / 2,
      prng         = prng,
      position     = lbrToCartesian(ctx, Vector.create(218, 53.5, 28.6)),
      velocity     = Vector.create(-156, 79, 107),
      comp1        = Dwarf.plummer{ mass = massL, scaleLength = rscaleL },
      comp2        = Dwarf.plummer{ mass = massD, scaleLength = rscaleD },
      ignore       = true
   }
end

function makeHistogram()
   return HistogramParams.create{
      phi = 128.79, theta = 54.39, psi = 90.70,
      lambdaStart = -150, lambdaEnd = 150, lambdaBins = 50,
      betaStart = -15, betaEnd = 15, betaBins = 1
   }
end
