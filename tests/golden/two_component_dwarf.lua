-- Two-component dwarf for the initial-condition checks: the reference's mixed-dwarf sampler
-- (predefinedModels.mixeddwarf with two Dwarf components, by default Dwarf.plummer as the sample
-- workunit nbody/sample_workunits/for_developers.lua builds it) placed at a fixed position and
-- velocity, without the reverse orbit, so that only the sampler is exercised.
-- Arguments: nbody, nbody_baryon, mass_l, rscale_l, mass_d, rscale_d, and optionally
-- type_l, type_d (plummer, nfw, general_hernquist or cored) and r1, rc (of cored components).

arg = {...}

assert(argSeed ~= nil, "seed argument missing")
prng = DSFMT.create(argSeed)

nbody = tonumber(arg[1])
nbodyBaryon = tonumber(arg[2])
massL = tonumber(arg[3])
rscaleL = tonumber(arg[4])
massD = tonumber(arg[5])
rscaleD = tonumber(arg[6])
typeL = arg[7] or "plummer"
typeD = arg[8] or "plummer"
coreR1 = tonumber(arg[9] or "0")
coreRc = tonumber(arg[10] or "0")

local function component(kind, m, a)
   if kind == "cored" then
      return Dwarf.cored{ mass = m, scaleLength = a, r1 = coreR1, rc = coreRc }
   end
   return Dwarf[kind]{ mass = m, scaleLength = a }
end

function makePotential()
   return Potential.create{
      spherical = Spherical.hernquist{ mass = 1.52954402E5, scale = 0.7 },
      disk      = Disk.miyamotoNagai{ mass = 4.45865888E5, scaleLength = 6.5, scaleHeight = 0.26 },
      disk2     = Disk.none{ mass = 3.0e5 },
      halo      = Halo.logarithmic{ vhalo = 73, scaleLength = 12, flattenZ = 1 }
   }
end

function makeContext()
   return NBodyCtx.create{
      timestep   = 1.0e-4,
      timeEvolve = 1.0e-3,
      eps2       = 1.0e-6,
      criterion  = "TreeCode",
      useQuad    = true,
      theta      = 0.5,
      BetaSigma  = 2.5,
      VelSigma   = 2.5,
      DistSigma  = 2.5,
      PMSigma    = 2.5,
      BetaCorrect = 1.111,
      VelCorrect = 1.111,
      DistCorrect = 1.111,
      PMCorrect  = 1.111,
      IterMax    = 6
   }
end

function makeBodies(ctx, potential)
   local comp1 = component(typeL, massL, rscaleL)
   local comp2 = component(typeD, massD, rscaleD)
   return predefinedModels.mixeddwarf{
      nbody        = nbody,
      nbody_baryon = nbodyBaryon,
      prng         = prng,
      position     = Vector.create(-21.6, -10.4, 23.2),
      velocity     = Vector.create(-150.0, 80.0, 100.0),
      comp1        = comp1,
      comp2        = comp2,
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
