#= LBMengineB200.jl — Julia front end of liblbm_b200.so (B200 lattice-Boltzmann time step).

Drop-in for the time-step path of LBMengine.jl's GPU module: the same
`modelInit`, `addSquirmer!`, `addBead!`, `LBMpropagate!`, `hydroVariablesUpdate!`
names and keywords (src/LBMengine.jl:27-41), with every tick computed by the
CUDA library through `ccall`.  Keyword resolution follows
src/gpu/initMethods.jl:440-702 (modelInit) and :91-222 (addSquirmer!).

The library path is taken from ENV["LBM_B200_LIB"] or defaults to the
in-tree build next to this directory.
=#
module LBMengineB200

export LBMmodel, modelInit, addBead!, addSquirmer!, LBMpropagate!, hydroVariablesUpdate!, viscousStressTensor,
       addLinearBond!, addPolarBond!, addBistableBond!, addDipoles!, addLennardJones!, addWCA!, writeTrajectories

const LIB = get(ENV, "LBM_B200_LIB", joinpath(@__DIR__, "..", "liblbm_b200.so"))

# ---- C structs (include/lbm_b200.h) --------------------------------------
struct LbmConfig
    dims::Int32; lattice::Int32; n::NTuple{3,Int64}; coords::NTuple{3,Ptr{Float64}}
    x0::NTuple{3,Float64}; dx::Float64; tau::Float64; tau_minus::Float64
    collision::Int32; compressible::Int32; force_mode::Int32; storage::Int32
    force::NTuple{3,Float64}; force_field::Ptr{Float64}; wall_mask::Ptr{UInt8}
    wall_velocity::Ptr{Float64}; rho_init::Ptr{Float64}; u_init::Ptr{Float64}
    rho_uniform::Float64; u_uniform::NTuple{3,Float64}; rho_ref::Float64; store_scale::Float64
    device::Int32; schedule::Int32; particle_rules::Int32; rounding::Int32
end

struct LbmParticleParams
    kind::Int32; couple_forces::Int32; couple_torques::Int32; reserved::Int32
    radius::Float64; mass_density::Float64
    position::NTuple{3,Float64}; velocity::NTuple{3,Float64}; angular_velocity::NTuple{3,Float64}
    swimming_direction::NTuple{3,Float64}; B1::Float64; B2::Float64
end

struct LbmParticleState
    id::Int32; kind::Int32; couple_forces::Int32; couple_torques::Int32
    radius::Float64; inverse_mass::Float64; inverse_inertia::Float64; B1::Float64; B2::Float64
    position::NTuple{3,Float64}; velocity::NTuple{3,Float64}; angular_velocity::NTuple{3,Float64}
    swimming_direction::NTuple{3,Float64}; last_force::NTuple{3,Float64}; last_torque::NTuple{3,Float64}
end

struct LbmInteraction
    kind::Int32; id1::Int32; id2::Int32; id3::Int32; p::NTuple{4,Float64}
end

struct LbmInfo
    dims::Int32; lattice::Int32; q::Int32; storage::Int32
    n::NTuple{3,Int64}; cells::Int64; tick::Int64; time::Float64
    num_particles::Int32; bytes_per_population::Int32; device_bytes::Int64
    bulk_kernel::Int32; bulk_threads::Int32; bulk_stages::Int32; reserved::Int32
end

lastError(h::Ptr{Cvoid}) = unsafe_string(ccall((:lbm_last_error, LIB), Cstring, (Ptr{Cvoid},), h))
globalError() = unsafe_string(ccall((:lbm_last_global_error, LIB), Cstring, ()))

function check(code::Integer, h::Ptr{Cvoid}=C_NULL)
    code == 0 && return nothing
    msg = h == C_NULL ? globalError() : lastError(h)
    code == -1 ? throw(AssertionError(msg)) : error("lbm_b200 error $code: $msg")
end

mutable struct LBMmodel
    handle::Ptr{Cvoid}
    dims::Int
    q::Int
    shape::Tuple
    spaceTime::NamedTuple
    fluidParams::NamedTuple
    schemes::Vector{Symbol}
    keep::Vector{Any}          # arrays the C config points into
    particleInteractions::Vector{Any}
    function LBMmodel(h, dims, q, shape, spaceTime, fluidParams, schemes, keep)
        m = new(h, dims, q, shape, spaceTime, fluidParams, schemes, keep, Any[])
        finalizer(mm -> (mm.handle != C_NULL && ccall((:lbm_destroy, LIB), Cvoid, (Ptr{Cvoid},), mm.handle);
                          mm.handle = C_NULL), m)
        return m
    end
end

const VSETS = Dict(:D2Q9 => (2, 9), :D3Q15 => (3, 15), :D3Q19 => (3, 19), :D3Q27 => (3, 27))

"modelInit(; ...) — keyword resolution of src/gpu/initMethods.jl:440-702, state on the GPU."
function modelInit(; massDensity = :default, fluidVelocity = :default, velocities = :default,
                   collisionModel = :default, relaxationTimeRatio = :default, viscosity = :default,
                   timeStep = :default, latticeParameter = :default, kineticParameter = 0.25,
                   xlims = :default, ylims = :default, zlims = :default, dims = 2,
                   walledDimensions = :default, walls = :default, movingWalls = :default,
                   isFluidCompressible = true, forceDensity = :default, storage = :f32, device = -1,
                   particleRules = :gpu, rounding = :stochastic, saveData = false)
    @assert any(x -> x == :default, [timeStep, relaxationTimeRatio, viscosity]) "timeStep, relaxationTimeRatio, and viscosity cannot be all simultaneously defined!"
    @assert any(x -> x == :default, [timeStep, latticeParameter]) "timeStep, and latticeParameter cannot be both simultaneously defined!"
    latticeParameter != :default && (timeStep = latticeParameter)
    if timeStep == :default
        relaxationTimeRatio == :default && (relaxationTimeRatio = 15)
        viscosity == :default && (viscosity = 1)
        timeStep = 3 * viscosity / (relaxationTimeRatio - 0.5)
    elseif relaxationTimeRatio == :default
        viscosity == :default && (viscosity = 1)
        relaxationTimeRatio = 3 * viscosity / timeStep + 0.5
    else
        viscosity = timeStep / 3 * (relaxationTimeRatio - 0.5)
    end
    dt = Float64(timeStep)
    xlims == :default && (xlims = (-1, 1)); ylims == :default && (ylims = xlims); zlims == :default && (zlims = xlims)
    axes = [collect(range(l[1], stop = l[2], step = dt)) for l in (xlims, ylims, zlims)[1:dims]]
    shape = Tuple(length.(axes))
    velocities == :default && (velocities = [:D1Q3, :D2Q9, :D3Q15][dims])
    vd, lattice = VSETS[velocities]
    @assert vd == dims "The chosen velocity must be $dims-dimensional!"
    collisionModel == :default && (collisionModel = :trt)
    @assert collisionModel in (:bgk, :trt) "Collision model $collisionModel is not implemented!"
    tau = relaxationTimeRatio * dt
    Λ = kineticParameter == :debug ? viscosity^2 / (dt^2 / 9) : kineticParameter
    tau_minus = collisionModel == :trt ? Λ * dt^2 / 3 / viscosity + dt / 2 : 0.0
    keep = Any[axes...]
    wall = nothing
    if walledDimensions != :default && !isempty(walledDimensions)
        wall = zeros(UInt8, shape)
        for a in walledDimensions
            idx = [1:s for s in shape]; idx[a] = 1:1; wall[idx...] .= 1
            idx[a] = shape[a]:shape[a]; wall[idx...] .= 1
        end
    end
    if walls != :default
        g = dims == 2 ? [walls(x, y) for x in axes[1], y in axes[2]] : [walls(x, y, z) for x in axes[1], y in axes[2], z in axes[3]]
        wall = wall === nothing ? UInt8.(g) : (wall .| UInt8.(g))
    end
    uw = nothing
    if movingWalls != :default
        vals = dims == 2 ? [movingWalls(x, y) for x in axes[1], y in axes[2]] : [movingWalls(x, y, z) for x in axes[1], y in axes[2], z in axes[3]]
        uw = zeros(Float64, shape..., dims)
        for k in 1:dims; selectdim(uw, dims + 1, k) .= getindex.(vals, k); end
        wall === nothing && (wall = zeros(UInt8, shape))
    end
    fmode, fvec, ffield = 0, (0.0, 0.0, 0.0), nothing
    if forceDensity != :default
        if forceDensity isa AbstractVector && length(forceDensity) == dims
            fmode = 1; fvec = Tuple(Float64[forceDensity; zeros(3 - dims)])
        else
            fmode = 2; ffield = Array{Float64}(forceDensity)
        end
    end
    rho_ptr = C_NULL; rho_u = 1.0
    if massDensity isa Number
        rho_u = Float64(massDensity)
    elseif massDensity != :default
        rhoa = Array{Float64}(massDensity); push!(keep, rhoa); rho_ptr = pointer(rhoa)
    end
    u_ptr = C_NULL; u_u = (0.0, 0.0, 0.0)
    if fluidVelocity != :default
        if ndims(fluidVelocity) == 1
            u_u = Tuple(Float64[fluidVelocity; zeros(3 - dims)])
        else
            ua = Array{Float64}(fluidVelocity); push!(keep, ua); u_ptr = pointer(ua)
        end
    end
    wall !== nothing && push!(keep, wall); uw !== nothing && push!(keep, uw); ffield !== nothing && push!(keep, ffield)
    store = Dict(:f32 => 0, :f16 => 1, :bf16 => 2, :f64 => 3)[storage]
    cfg = LbmConfig(dims, lattice, (Int64.((shape..., ones(Int, 3 - dims)...))...,),
                    ntuple(a -> a <= dims ? pointer(axes[a]) : Ptr{Float64}(C_NULL), 3),
                    ntuple(a -> a <= dims ? axes[a][1] : 0.0, 3), dt, tau, tau_minus,
                    collisionModel == :bgk ? 0 : 1, isFluidCompressible ? 1 : 0, fmode, store, fvec,
                    ffield === nothing ? C_NULL : pointer(ffield), wall === nothing ? C_NULL : pointer(wall),
                    uw === nothing ? C_NULL : pointer(uw), rho_ptr, u_ptr, rho_u, u_u, 0.0, 0.0, device, 0,
                    particleRules == :cpu ? 1 : 0, rounding == :nearest ? 1 : 0)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve keep check(ccall((:lbm_create, LIB), Cint, (Ref{LbmConfig}, Ref{Ptr{Cvoid}}), cfg, h))
    schemes = Symbol[collisionModel]
    wall !== nothing && push!(schemes, :bounceBack)
    uw !== nothing && push!(schemes, :movingWalls)
    fmode != 0 && push!(schemes, :guo)
    saveData && push!(schemes, :saveData)
    spaceTime = (; coordinates = Tuple(axes), latticeParameter = dt, timeStep = dt, latticeSpeed = 1.0, dims)
    fluidParams = (; relaxationTime = tau, viscosity, relaxationTimePlus = tau, relaxationTimeMinus = tau_minus)
    model = LBMmodel(h[], dims, lattice, shape, spaceTime, fluidParams, schemes, keep)
    if saveData  # src/gpu/initMethods.jl:671-675 and :698
        rm("output.lbm"; force = true, recursive = true)
        mkdir("output.lbm")
        writeTrajectories(model)
        check(ccall((:lbm_output_flush, LIB), Cint, (Ptr{Cvoid},), model.handle), model.handle)
    end
    return model
end

function _add!(model::LBMmodel, p::LbmParticleParams)
    id = Ref{Int32}(0)
    check(ccall((:lbm_add_particle, LIB), Cint, (Ptr{Cvoid}, Ref{LbmParticleParams}, Ref{Int32}), model.handle, p, id), model.handle)
    for s in (:ladd, :bounceBack); s in model.schemes || push!(model.schemes, s); end
    if :saveData in model.schemes  # writeParticleTrajectory of the new particle (initMethods.jl:86, 219)
        q = model.particles[id[]]
        _appendParticleRows(model.dims, [(model.tick, model.time, id[], q.position, q.velocity, q.angularVelocity)])
    end
    return nothing
end

# ---- :saveData output (src/gpu/aux.jl:271-356, src/gpu/fluids.jl:243-259) --------
"writeTrajectories(model): output.lbm/fluidTrj_<tick>.csv, formatted and written by the library's host thread."
writeTrajectories(model::LBMmodel) =
    check(ccall((:lbm_write_fluid_csv, LIB), Cint, (Ptr{Cvoid}, Cstring), model.handle,
                "output.lbm/fluidTrj_$(model.tick).csv"), model.handle)

function _appendParticleRows(d, rows)
    path = "output.lbm/particlesTrj.csv"
    header = d == 2 ? "tick,time,particleId,position_x,position_y,velocity_x,velocity_y,angularVelocity" :
             "tick,time,particleId,position_x,position_y,position_z,velocity_x,velocity_y,velocity_z," *
             "angularVelocity_x,angularVelocity_y,angularVelocity_z"
    new = !isfile(path)
    open(path, "a") do io
        new && println(io, header)
        for (tick, time, id, R, v, w) in rows
            println(io, join(string.([tick; time; id; R[1:d]; v[1:d]; d == 2 ? w[1] : w[1:3]]), ","))
        end
    end
end

const RING_TICKS = 1024

function _propagateSaving!(model::LBMmodel, n::Integer, ticksSaved)
    ticksSaved == :default && (ticksSaved = 100)
    dt = model.spaceTime.timeStep
    t0 = model.tick
    totalTicks = floor(n * dt / dt)
    checkpoints = range(t0, stop = t0 + totalTicks, length = ticksSaved) |> collect .|> round .|> Int64
    np = length(model.particles); d = model.dims
    h = model.handle
    np > 0 && check(ccall((:lbm_record_trajectories, LIB), Cint, (Ptr{Cvoid}, Int64), h, RING_TICKS), h)
    done = 0; time = model.time
    try
        while done < n
            nxt = minimum([[c - t0 for c in checkpoints if c - t0 > done]; n])
            seg = min(nxt - done, RING_TICKS)
            check(ccall((:lbm_step, LIB), Cint, (Ptr{Cvoid}, Int64), h, seg), h)
            tick0 = t0 + done; done += seg
            if np > 0
                buf = zeros(Float64, 9, np, seg); got = Ref{Int64}(0)
                check(ccall((:lbm_read_trajectories, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64, Ref{Int64}),
                            h, buf, seg, got), h)
                rows = Any[]
                for t in 1:seg
                    time += dt
                    for p in 1:np
                        r = buf[:, p, t]
                        push!(rows, (tick0 + t, time, p, r[1:3], r[4:6], r[7:9]))
                    end
                end
                _appendParticleRows(d, rows)
            end
            model.tick in checkpoints && writeTrajectories(model)
        end
    finally
        np > 0 && ccall((:lbm_record_trajectories, LIB), Cint, (Ptr{Cvoid}, Int64), h, 0)
        check(ccall((:lbm_output_flush, LIB), Cint, (Ptr{Cvoid},), h), h)
    end
    return nothing
end

# ---- particle interactions (src/gpu/initMethods.jl:224-414) -------------------
function _pushInteractions!(model::LBMmodel, t = model.time)
    items = LbmInteraction[]
    for it in model.particleInteractions
        if it.kind in (:linear, :bistable, :polar)
            k = Dict(:linear => 0, :bistable => 1, :polar => 2)[it.kind]
            p = Tuple(Float64[it.params; zeros(4 - length(it.params))])
            push!(items, LbmInteraction(k, it.id1, it.id2, it.kind == :polar ? it.id3 : 0, p))
        else
            B = it.kind == :dipole ? Float64.(it.magneticField isa Function ? it.magneticField(t) : it.magneticField) : Float64[]
            p = it.kind == :dipole ? (it.dipoleConstant, [B; zeros(3 - length(B))]...) : (it.epsilon, it.sigma, it.cutoff, 0.0)
            for (a, b) in it.pairs
                push!(items, LbmInteraction(it.kind == :dipole ? 4 : 3, a, b, 0, p))
            end
        end
    end
    check(ccall((:lbm_set_interactions, LIB), Cint, (Ptr{Cvoid}, Ptr{LbmInteraction}, Int32), model.handle, items,
                length(items)), model.handle)
end

_dist(model, i, j) = sqrt(sum(abs2, model.particles[j].position - model.particles[i].position))
_pairs(ids) = [(ids[i], ids[j]) for i in eachindex(ids) for j in eachindex(ids) if i < j]

"addLinearBond!(model, id1, id2; ...) — src/gpu/initMethods.jl:229-246."
function addLinearBond!(model::LBMmodel, id1::Int, id2::Int; equilibriumDisplacement = :default, stiffness = 1)
    equilibriumDisplacement == :default && (equilibriumDisplacement = _dist(model, id1, id2))
    @assert equilibriumDisplacement isa Number "equilibriumDisplacement must be a number!"
    @assert stiffness isa Number "stiffness must be a number!"
    push!(model.particleInteractions, (; kind = :linear, id1, id2, params = [equilibriumDisplacement, stiffness]))
    _pushInteractions!(model)
end

"addPolarBond!(model, id1, id2, id3; ...) — src/gpu/initMethods.jl:248-274."
function addPolarBond!(model::LBMmodel, id1::Int, id2::Int, id3::Int; equilibriumAngle = :default, stiffness = 1)
    P = model.particles
    vecA = P[id1].position - P[id2].position; vecB = P[id3].position - P[id2].position
    cosAlpha = sum(vecA .* vecB) / (sqrt(sum(abs2, vecA)) * sqrt(sum(abs2, vecB)))
    equilibriumAngle == :default && (equilibriumAngle = acos(cosAlpha))
    @assert equilibriumAngle isa Number "equilibriumAngle must be a number!"
    @assert stiffness isa Number "stiffness must be a number!"
    push!(model.particleInteractions, (; kind = :polar, id1, id2, id3, params = [equilibriumAngle, stiffness]))
    _pushInteractions!(model)
end

"addBistableBond!(model, id1, id2; ...) — src/gpu/initMethods.jl:283-309."
function addBistableBond!(model::LBMmodel, id1::Int, id2::Int; lowDisp = :default, highDisp = :default, hillHeight = 1)
    lowDisp == :default && (lowDisp = _dist(model, id1, id2))
    highDisp == :default && (highDisp = lowDisp + model.spaceTime.latticeParameter)
    trapRadius = (highDisp + lowDisp) / 2; trapWidth = highDisp - lowDisp
    push!(model.particleInteractions, (; kind = :bistable, id1, id2,
                                       params = [trapRadius, 4 * 16 * hillHeight / trapWidth^4, 2 * 8 * hillHeight / trapWidth^2]))
    _pushInteractions!(model)
end

"addDipoles!(model, ids...; ...) — src/gpu/initMethods.jl:317-360."
function addDipoles!(model::LBMmodel, ids...; magneticField = [1, 0], susceptibility = 0.5, permeability = 400 * pi,
                     rewrite = false)
    ids = isempty(ids) ? collect(eachindex(model.particles)) : collect(ids)
    k = findfirst(it -> it.kind == :dipole, model.particleInteractions)
    if k !== nothing && !rewrite
        ids = sort(unique([ids; [i for p in model.particleInteractions[k].pairs for i in p]]))
    end
    @assert length(ids) > 1 "There must be at least two dipoles!"
    r = model.particles[ids[1]].particleParams.radius
    new = (; kind = :dipole, pairs = _pairs(ids), dipoleConstant = 4 * pi * r^6 * susceptibility^2 / (3 * permeability),
           magneticField)
    if k === nothing || rewrite
        k !== nothing && deleteat!(model.particleInteractions, k)
        push!(model.particleInteractions, new)
    else
        model.particleInteractions[k] = merge(model.particleInteractions[k], (; pairs = new.pairs))
    end
    _pushInteractions!(model)
end

function _defaultEpsilon(model)
    rho = filter(x -> !(x ≈ 0), model.massDensity)
    return sum(rho) / length(rho) * model.spaceTime.latticeParameter^5 / model.spaceTime.timeStep^2
end

"addLennardJones!(model; ...) — src/gpu/initMethods.jl:362-397."
function addLennardJones!(model::LBMmodel; epsilon = :default, sigma = :default, cutoff = :default)
    k = findfirst(it -> it.kind == :lennardJones, model.particleInteractions)
    k !== nothing && deleteat!(model.particleInteractions, k)
    epsilon == :default && (epsilon = _defaultEpsilon(model))
    sigma == :default && (sigma = 2 * model.particles[1].particleParams.radius + model.spaceTime.latticeParameter)
    cutoff == :default && (cutoff = Inf)
    push!(model.particleInteractions, (; kind = :lennardJones, pairs = _pairs(collect(eachindex(model.particles))),
                                       epsilon, sigma, cutoff))
    _pushInteractions!(model)
end

"addWCA!(model; ...) — src/gpu/initMethods.jl:399-413."
function addWCA!(model::LBMmodel; epsilon = :default, sigma = :default)
    epsilon == :default && (epsilon = _defaultEpsilon(model))
    sigma == :default && (sigma = 2 * model.particles[1].particleParams.radius + model.spaceTime.latticeParameter)
    addLennardJones!(model; epsilon, sigma, cutoff = 2^(1 / 6) * sigma)
end

"viscousStressTensor(model) — src/cpu/fluids.jl:507-520: a dims x dims matrix of fields."
function viscousStressTensor(model::LBMmodel)
    d = model.dims
    s = zeros(Float64, model.shape..., d, d)
    check(ccall((:lbm_get_stress, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}), model.handle, s), model.handle)
    return [selectdim(selectdim(s, d + 2, b), d + 1, a) |> copy for a in 1:d, b in 1:d]
end

pad3(v) = Tuple(Float64[collect(v); zeros(3 - length(v))])

"addSquirmer!(model; ...) — keyword resolution of src/gpu/initMethods.jl:91-173."
function addSquirmer!(model::LBMmodel; massDensity = 1.0, radius = 0.1, position = :default, velocity = :default,
                      angularVelocity = :default, slipSpeed = :default, swimmingSpeed = :default,
                      swimmingDirection = :default, B1 = :default, B2 = :default, beta = :default,
                      coupleTorques = false, coupleForces = false)
    d = model.dims
    position == :default && (position = zeros(d)); velocity == :default && (velocity = zeros(d))
    angularVelocity == :default && (angularVelocity = d == 2 ? 0.0 : zeros(3))
    @assert any(x -> x == :default, [B1, B2, beta]) "B1, B2, and beta cannot be all simultaneously defined!"
    if beta == :default
        B1 == :default && (B1 = 1); B2 == :default && (B2 = 0); beta = B2 / B1
    elseif B2 == :default
        B1 == :default && (B1 = 1); B2 = B1 * beta
    else
        @assert beta != 0 "if beta = 0, then B2 can only be zero! In this case, do not declare both."
        B1 = B2 / beta
    end
    swimmingDirection == :default && (swimmingDirection = [1.0; zeros(d - 1)])
    e = swimmingDirection ./ sqrt(sum(abs2, swimmingDirection))
    @assert any(x -> x == :default, [slipSpeed, swimmingSpeed]) "slipSpeed and swimmingSpeed cannot be all simultaneously defined!"
    if slipSpeed == :default
        swimmingSpeed == :default && (swimmingSpeed = 1e-3)
        e = e .* sign(swimmingSpeed); B1 = abs(3 / 2 * swimmingSpeed); B2 = B1 * beta
    else
        nf = maximum(abs((B1 + B2 * cos(t)) * sin(t)) for t in range(-pi, stop = pi, length = 100))
        B1 *= slipSpeed / nf; B2 *= slipSpeed / nf
    end
    w = d == 2 ? (Float64(angularVelocity), 0.0, 0.0) : pad3(angularVelocity)
    _add!(model, LbmParticleParams(1, coupleForces, coupleTorques, 0, radius, massDensity, pad3(position),
                                   pad3(velocity), w, pad3(e), B1, B2))
end

"addBead!(model; ...) — src/gpu/initMethods.jl:7-89."
function addBead!(model::LBMmodel; massDensity = 1.0, radius = 0.1, position = :default, velocity = :default,
                  angularVelocity = :default, coupleTorques = false, coupleForces = false)
    d = model.dims
    position == :default && (position = zeros(d)); velocity == :default && (velocity = zeros(d))
    angularVelocity == :default && (angularVelocity = d == 2 ? 0.0 : zeros(3))
    w = d == 2 ? (Float64(angularVelocity), 0.0, 0.0) : pad3(angularVelocity)
    _add!(model, LbmParticleParams(0, coupleForces, coupleTorques, 0, radius, massDensity, pad3(position),
                                   pad3(velocity), w, (0.0, 0.0, 0.0), 0.0, 0.0))
end

"LBMpropagate!(model; ticks | simulationTime, ticksSaved) — src/gpu/fluids.jl:228-264."
function LBMpropagate!(model::LBMmodel; simulationTime = :default, ticks = :default, verbose = false,
                       ticksSaved = :default)
    @assert any(x -> x == :default, [simulationTime, ticks]) "simulationTime and ticks cannot be simultaneously chosen, as the time step is defined already in the model!"
    dt = model.spaceTime.timeStep
    n = simulationTime == :default && ticks == :default ? 100 :
        ticks == :default ? length(range(dt, stop = simulationTime, step = dt)) : ticks
    timeField = any(it -> it.kind == :dipole && it.magneticField isa Function, model.particleInteractions)
    if timeField  # B(t) of the dipoles at each tick's time (molecularDynamicsTick! runs after time += dt)
        for _ in 1:n
            _pushInteractions!(model, model.time + dt)
            check(ccall((:lbm_step, LIB), Cint, (Ptr{Cvoid}, Int64), model.handle, 1), model.handle)
        end
    elseif :saveData in model.schemes
        _propagateSaving!(model, n, ticksSaved)
    else
        check(ccall((:lbm_step, LIB), Cint, (Ptr{Cvoid}, Int64), model.handle, n), model.handle)
    end
    verbose && println("\r t = ", round(n * dt; digits = 2))
    return nothing
end

"The library keeps rho and u consistent with the populations; kept for API compatibility."
hydroVariablesUpdate!(model::LBMmodel; useEquilibriumScheme = false) = nothing

function Base.getproperty(m::LBMmodel, s::Symbol)
    if s === :massDensity || s === :fluidVelocity
        N = prod(getfield(m, :shape)); d = getfield(m, :dims)
        rho = zeros(Float64, getfield(m, :shape)); u = zeros(Float64, getfield(m, :shape)..., d)
        check(ccall((:lbm_get_fields, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}),
                    getfield(m, :handle), rho, u), getfield(m, :handle))
        return s === :massDensity ? rho : u
    elseif s === :distributions
        f = zeros(Float64, getfield(m, :shape)..., getfield(m, :q))
        check(ccall((:lbm_get_distributions, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}), getfield(m, :handle), f),
              getfield(m, :handle))
        return f
    elseif s === :particles
        cnt = Ref{Int32}(0)
        check(ccall((:lbm_get_particles, LIB), Cint, (Ptr{Cvoid}, Ptr{LbmParticleState}, Int32, Ref{Int32}),
                    getfield(m, :handle), C_NULL, 0, cnt), getfield(m, :handle))
        st = Vector{LbmParticleState}(undef, cnt[])
        check(ccall((:lbm_get_particles, LIB), Cint, (Ptr{Cvoid}, Ptr{LbmParticleState}, Int32, Ref{Int32}),
                    getfield(m, :handle), st, cnt[], cnt), getfield(m, :handle))
        d = getfield(m, :dims)
        return [(; id = p.id, position = collect(p.position[1:d]), velocity = collect(p.velocity[1:d]),
                  angularVelocity = d == 2 ? p.angular_velocity[1] : collect(p.angular_velocity),
                  particleParams = (; radius = p.radius, B1 = p.B1, B2 = p.B2,
                                    swimmingDirection = collect(p.swimming_direction[1:d]),
                                    inverseMass = p.inverse_mass, inverseMomentOfInertia = p.inverse_inertia))
                for p in st]
    elseif s === :tick || s === :time
        info = Ref{LbmInfo}()
        check(ccall((:lbm_get_info, LIB), Cint, (Ptr{Cvoid}, Ref{LbmInfo}), getfield(m, :handle), info),
              getfield(m, :handle))
        return s === :tick ? info[].tick : info[].time
    end
    return getfield(m, s)
end

end # module
