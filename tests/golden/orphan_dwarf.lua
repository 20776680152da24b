-- Single-Plummer dwarfs on Orphan-stream orbits: the set-ups of the reference's golden
-- likelihood tests (nbody/tests/orphan_models/model_*.lua, driven by
-- nbody/tests/RunTestUnits.lua), restated as one table of variants for this repository's
-- golden checks.
-- Arguments: nbody, variant (a key of `variants` below; default "5"), options.
--   variant "4", "5", "5b" (model_5_bounds_test), "6", "8", "9", "ninkovic", "triaxial",
--   "newhist1".."newhist3", "bar", "LMC", "LMC_bar"; each entry records its potential, dwarf,
--   orbit and the context fields that differ between the models.
--   options (optional): "allterms" turns on every comparison of the likelihood (velocity
--   dispersion, line-of-sight velocity, beta average, distance, proper motions); "bestlike"
--   turns on the best-likelihood scan over the last 5% of the steps; "betaN" (N a number)
--   gives the histogram N beta bins instead of one (a two-dimensional histogram).
-- The seed comes from the command line (argSeed), as in the reference tests.

arg = {...}

seed = argSeed
nbody = arg[1]
local variantName = arg[2] or "5"
local options = arg[3] or ""
local allTerms = string.find(options, "allterms") ~= nil
local bestLike = string.find(options, "bestlike") ~= nil
local betaBins = tonumber(string.match(options, "beta(%d+)") or "1")

assert(seed ~= nil, "seed argument missing")
assert(nbody ~= nil, "body count argument missing")

prng = DSFMT.create(seed)

-- potential components, built on demand
local function hernquist(m, a) return function() return Spherical.hernquist{ mass = m, scale = a } end end
local function plummer(m, a) return function() return Spherical.plummer{ mass = m, scale = a } end end
local function mn(m, a, b)
   return function() return Disk.miyamotoNagai{ mass = m, scaleLength = a, scaleHeight = b } end
end
local function logHalo(v, d, q)
   return function() return Halo.logarithmic{ vhalo = v, scaleLength = d, flattenZ = q } end
end

local windowStart = 0.95          -- the bar model's best-likelihood window starts here

local variants = {
   ["4"] = { bulge = hernquist(1.52954402E5, 0.7), disk = mn(4.45865888E5, 6.5, 0.26),
             halo = logHalo(114, 12, 1), eps2Kind = 1, r = 28.9, v = { -179, 106, 109 } },
   ["5"] = { bulge = plummer(1.52954402E5, 0.7), disk = mn(4.45865888E5, 6.5, 0.26),
             halo = logHalo(73, 12, 1), eps2Kind = 1, r = 28.6, v = { -156, 79, 107 } },
   ["5b"] = { bulge = plummer(1.52954402E5, 0.7), disk = mn(4.45865888E5, 6.5, 0.26),
              halo = logHalo(73, 12, 1), eps2Kind = 1, r = 28.6, v = { -156, 79, 107 },
              dwarfMass = 1, dwarfRadius = 0.05, timeEvolve = 4.132339410448132,
              tstop = 4.291337464901487 },
   ["6"] = { bulge = plummer(1.52954402E5, 0.7), disk = mn(4.45865888E5, 6.5, 0.26),
             halo = function() return Halo.nfw{ vhalo = 155, scaleLength = 22.25 } end,
             eps2Kind = 0, r = 28.9, v = { -178, 106, 108 } },
   ["8"] = { bulge = plummer(4.0373214139267E4, 0.249), disk = mn(3.2340408839019E5, 3.67, 0.305),
             halo = function()
                return Halo.allenSantillan{ mass = 4.7276406194167E4, scaleLength = 1.52,
                                            lambda = 200.0, gamma = 2.0 }
             end,
             eps2Kind = 0, r = 28.9, v = { -179, 106, 109 } },
   ["9"] = { bulge = plummer(14852.322299938, 0.25), disk = mn(285750.313545277, 5.16, 0.311),
             halo = function()
                return Halo.wilkinsonEvans{ mass = 2570079.320803279, scaleLength = 64.3 }
             end,
             eps2Kind = 1, r = 28.9, v = { -179, 106, 109 } },
   ["ninkovic"] = { bulge = hernquist(1.52954402E5, 0.7), disk = mn(4.45865888E5, 6.5, 0.26),
                    halo = function()
                       return Halo.ninkovic{ rho0 = 23.6, scaleLength = 17.0, lambda = 93.6 }
                    end,
                    eps2Kind = 0, r = 28.9, v = { -179, 106, 109 } },
   ["triaxial"] = { bulge = hernquist(1.52954402E5, 0.7), disk = mn(4.45865888E5, 6.5, 0.26),
                    halo = function()
                       return Halo.triaxial{ vhalo = 116, scaleLength = 16.3, flattenZ = 1.43,
                                             flattenX = 1.26, flattenY = 1.0, triaxAngle = 96 }
                    end,
                    eps2Kind = 1, r = 29.5, v = { -183, 101, 107 } },
   ["bar"] = { bulge = hernquist(1.52954402e5, 0.7), disk = mn(4.18972480e5, 6.5, 0.26),
               disk2 = function()
                  return Disk.orbitingBar{ mass = 2.689340798e4, scaleLength = 5.4,
                                           patternSpeed = 250.61, startAngle = 0.488692 }
               end,
               halo = logHalo(74.61, 12.0, 1.0), eps2Kind = 0, r = 28.8, v = { -170, 94, 108 },
               -- evolve to the end of the best-likelihood window, scan from its start, and
               -- calibrate the bar's phase with two more runs
               timeEvolve = (2.0 - windowStart) * 3.945, timeBack = 3.945,
               useBestLike = true, bestLikeStart = windowStart / (2.0 - windowStart),
               calibrationRuns = 2 },
   -- the LMC as a moving Plummer sphere with dynamical friction (reverseOrbit_LMC below)
   ["LMC"] = { bulge = hernquist(67479.9, 0.6), disk = mn(224933, 4, 0.26),
               halo = logHalo(155, 22.25, 1.1), eps2Kind = 1, r = 28.8, v = { -170, 94, 108 },
               lmc = true },
   ["LMC_bar"] = { bulge = hernquist(67479.9, 0.6), disk = mn(198040, 4, 0.26),
                   disk2 = function()
                      return Disk.orbitingBar{ mass = 2.689340798e4, scaleLength = 5.4,
                                               patternSpeed = 250.61, startAngle = 0.488692 }
                   end,
                   halo = logHalo(155, 22.25, 1.1), eps2Kind = 0, r = 28.8, v = { -170, 94, 108 },
                   lmc = true, timeBack = 3.945 },
}
local LMCMASS = 449865.888
local LMCSCALE = 15.0
-- newhist1..3: a 12-mass dwarf with the beta-average, line-of-sight and distance comparisons
local newhist = { { 1, 53.4, 28.7, { -158, 76, 108 } }, { 0, 53.6, 28.5, { -154, 78, 109 } },
                  { 1, 53.8, 28.9, { -159, 80, 105 } } }
for k, h in ipairs(newhist) do
   variants["newhist" .. k] = {
      bulge = plummer(152954.402000, 0.7), disk = mn(445865.888000, 6.5, 0.26),
      halo = logHalo(74.61, 12, 1), eps2Kind = h[1], b = h[2], r = h[3], v = h[4],
      dwarfMass = 12, newhist = true }
end

local V = variants[variantName]
assert(V ~= nil, "unknown variant " .. variantName)

dwarfMass = V.dwarfMass or 16
dwarfRadius = V.dwarfRadius or 0.2

function makePotential()
   return Potential.create{
      spherical = V.bulge(),
      disk      = V.disk(),
      disk2     = V.disk2 and V.disk2() or Disk.none{ mass = 3.0e5 },
      halo      = V.halo()
   }
end

function makeContext()
   local c = {
      timestep      = calculateTimestep(dwarfMass, dwarfRadius),
      timeEvolve    = V.timeEvolve or 3.945,
      eps2          = calculateEps2(nbody, dwarfRadius, V.eps2Kind),
      criterion     = "sw93",
      useQuad       = true,
      theta         = 1.0,
      BestLikeStart = V.bestLikeStart or 0.95,
      BetaSigma     = 2.5,
      VelSigma      = 2.5,
      DistSigma     = 2.5,
      PMSigma       = 2.5,
      BetaCorrect   = 1.111,
      VelCorrect    = 1.111,
      DistCorrect   = 1.111,
      PMCorrect     = 1.111,
      IterMax       = 6
   }
   if V.timeBack then c.timeBack = V.timeBack end
   if V.lmc then
      c.LMC = true
      c.LMCmass = LMCMASS
      c.LMCscale = LMCSCALE
      c.LMCDynaFric = true
   end
   if V.calibrationRuns then c.calibrationRuns = V.calibrationRuns end
   if V.useBestLike or bestLike then c.useBestLike = true end
   if V.newhist then
      c.b = V.b
      c.r = V.r
      c.vx = V.v[1]
      c.vy = V.v[2]
      c.vz = V.v[3]
      c.useBetaComp = true
      c.useVlos = true
      c.useDist = true
   end
   if allTerms then
      c.useVelDisp = true
      c.useBetaComp = true
      c.useVlos = true
      c.useDist = true
      c.usePropMot = true
   end
   return NBodyCtx.create(c)
end

function makeBodies(ctx, potential)
   local finalPosition, finalVelocity
   if V.lmc then
      finalPosition, finalVelocity = reverseOrbit_LMC{
         potential   = potential,
         position    = lbrToCartesian(ctx, Vector.create(218, 53.5, V.r)),
         velocity    = Vector.create(V.v[1], V.v[2], V.v[3]),
         LMCposition = Vector.create(-1.1, -41.1, -27.9),
         LMCvelocity = Vector.create(-57, -226, 221),
         LMCmass     = LMCMASS,
         LMCscale    = LMCSCALE,
         LMCDynaFric = true,
         coulomb_log = 0.470003629,
         ftime       = 4.5,
         tstop       = 4.0,
         dt          = ctx.timestep / 10.0
      }
   else
      finalPosition, finalVelocity = reverseOrbit{
         potential = potential,
         position  = lbrToCartesian(ctx, Vector.create(218, V.b or 53.5, V.r)),
         velocity  = Vector.create(V.v[1], V.v[2], V.v[3]),
         tstop     = V.tstop or 4.0,
         dt        = ctx.timestep / 10.0
      }
   end

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
      betaBins  = betaBins
   }
end
