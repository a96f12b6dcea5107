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

export LBMmodel, modelInit, addBead!, addSquirmer!, LBMpropagate!, hydroVariablesUpdate!

const LIB = get(ENV, "LBM_B200_LIB", joinpath(@__DIR__, "..", "liblbm_b200.so"))

# ---- C structs (include/lbm_b200.h) --------------------------------------
struct LbmConfig
    dims::Int32; lattice::Int32; n::NTuple{3,Int64}; coords::NTuple{3,Ptr{Float64}}
    x0::NTuple{3,Float64}; dx::Float64; tau::Float64; tau_minus::Float64
    collision::Int32; compressible::Int32; force_mode::Int32; storage::Int32
    force::NTuple{3,Float64}; force_field::Ptr{Float64}; wall_mask::Ptr{UInt8}
    wall_velocity::Ptr{Float64}; rho_init::Ptr{Float64}; u_init::Ptr{Float64}
    rho_uniform::Float64; u_uniform::NTuple{3,Float64}; rho_ref::Float64; store_scale::Float64
    device::Int32; schedule::Int32; particle_rules::Int32; reserved::Int32
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
    function LBMmodel(h, dims, q, shape, spaceTime, fluidParams, schemes, keep)
        m = new(h, dims, q, shape, spaceTime, fluidParams, schemes, keep)
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
                   particleRules = :gpu)
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
                    particleRules == :cpu ? 1 : 0, 0)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve keep check(ccall((:lbm_create, LIB), Cint, (Ref{LbmConfig}, Ref{Ptr{Cvoid}}), cfg, h))
    schemes = Symbol[collisionModel]
    wall !== nothing && push!(schemes, :bounceBack)
    uw !== nothing && push!(schemes, :movingWalls)
    fmode != 0 && push!(schemes, :guo)
    spaceTime = (; coordinates = Tuple(axes), latticeParameter = dt, timeStep = dt, latticeSpeed = 1.0, dims)
    fluidParams = (; relaxationTime = tau, viscosity, relaxationTimePlus = tau, relaxationTimeMinus = tau_minus)
    return LBMmodel(h[], dims, lattice, shape, spaceTime, fluidParams, schemes, keep)
end

function _add!(model::LBMmodel, p::LbmParticleParams)
    id = Ref{Int32}(0)
    check(ccall((:lbm_add_particle, LIB), Cint, (Ptr{Cvoid}, Ref{LbmParticleParams}, Ref{Int32}), model.handle, p, id), model.handle)
    for s in (:ladd, :bounceBack); s in model.schemes || push!(model.schemes, s); end
    return nothing
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

"LBMpropagate!(model; ticks | simulationTime) — src/gpu/fluids.jl:228-264."
function LBMpropagate!(model::LBMmodel; simulationTime = :default, ticks = :default, verbose = false)
    @assert any(x -> x == :default, [simulationTime, ticks]) "simulationTime and ticks cannot be simultaneously chosen, as the time step is defined already in the model!"
    dt = model.spaceTime.timeStep
    n = simulationTime == :default && ticks == :default ? 100 :
        ticks == :default ? length(range(dt, stop = simulationTime, step = dt)) : ticks
    check(ccall((:lbm_step, LIB), Cint, (Ptr{Cvoid}, Int64), model.handle, n), model.handle)
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
