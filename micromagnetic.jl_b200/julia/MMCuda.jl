# MMCuda.jl -- MicroMagnetic.jl binding of libmmcuda.so (B200, sm_100a).
#
# Loaded next to MicroMagnetic.jl, this module keeps the user API
# (FDMesh, Sim, set_Ms, init_m0, add_exch, add_dmi, add_anis, add_demag,
# add_zeeman, run_sim, run_until, relax) and routes the finite-difference hot
# path -- effective field, LLG right-hand side, RK4 / Dormand-Prince stepping
# and SD relaxation -- through the C ABI declared in include/mmcuda.h.
#
#   using MicroMagnetic, MMCuda
#   mesh = FDMesh(nx=256, ny=256, nz=64, dx=2e-9, dy=2e-9, dz=2e-9)
#   sim = Sim(mesh)                        # driver "LLG", DormandPrince
#   set_Ms(sim, 5.8e5); add_exch(sim, 1e-11); add_demag(sim)
#   init_m0(sim, (1, 0, 0))
#   MMCuda.attach!(sim; form=:fp32)        # copies state + terms to the GPU
#   run_sim(sim; steps=100, dt=1e-12)      # run_until -> mm_run_until
#
# attach! reads the term structs of src/head.jl (UniformExchange,
# SpatialExchange, BulkDMI, InterfacialDMI, Anisotropy, Zeeman, Demag) and
# replays them into the handle; the methods below then take precedence over
# the KernelAbstractions path for an attached Sim.
module MMCuda

using MicroMagnetic
import MicroMagnetic: effective_field, advance_step, run_until, relax, compute_system_energy

const libmmcuda = joinpath(@__DIR__, "..", "mmcuda", "libmmcuda.so")

struct MeshDesc
    nx::Int32; ny::Int32; nz::Int32
    dx::Float64; dy::Float64; dz::Float64
    pbc::Int32
end

mutable struct Stats
    t::Float64; step::Float64; step_next::Float64
    nsteps::Int64; nfevals::Int64; attempts::Int64; rejected::Int64
    status::Int32
end
Stats() = Stats(0, 0, 0, 0, 0, 0, 0, 0)

mutable struct Handle
    ptr::Ptr{Cvoid}
    n::Int
end

const HANDLES = IdDict{Any,Handle}()

function check(rc::Integer)
    rc == 0 && return nothing
    buf = Vector{UInt8}(undef, 1024)
    ccall((:mm_last_error, libmmcuda), Cint, (Ptr{UInt8}, Csize_t), buf, length(buf))
    msg = unsafe_string(pointer(buf))
    rc == -3 && throw(ErrorException("NaN: " * msg))
    error("libmmcuda error $rc: " * msg)
end

# AoS Float64 copies of arbitrary Float[] arrays (the ABI speaks Float64)
f64(a) = Vector{Float64}(Array(a))

"""
    attach!(sim::MicroSim; form=:fp64, device=0)

Create a libmmcuda handle for `sim` (MM_FP64 or MM_FP32 form), copy Ms, m,
pins, LLG parameters and the interaction terms into it.
"""
function attach!(sim::MicroMagnetic.MicroSim; form::Symbol=:fp64, device::Integer=0)
    mesh = sim.mesh
    pbc = Int32((mesh.xperiodic ? 1 : 0) | (mesh.yperiodic ? 2 : 0) | (mesh.zperiodic ? 4 : 0))
    d = Ref(MeshDesc(mesh.nx, mesh.ny, mesh.nz, mesh.dx, mesh.dy, mesh.dz, pbc))
    out = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:mm_create, libmmcuda), Cint, (Ref{MeshDesc}, Cint, Cint, Ref{Ptr{Cvoid}}),
                d, form == :fp32 ? 1 : 0, device, out))
    h = Handle(out[], sim.n_total)
    finalizer(x -> ccall((:mm_destroy, libmmcuda), Cint, (Ptr{Cvoid},), x.ptr), h)
    Ms = f64(sim.mu0_Ms) ./ MicroMagnetic.mu_0
    check(ccall((:mm_set_Ms, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}, Float64), h.ptr, Ms, 0.0))
    push_spin!(h, sim.spin)
    pins = UInt8.(Array(sim.pins))
    check(ccall((:mm_set_pins, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{UInt8}), h.ptr, pins))
    drv = sim.driver
    if drv isa MicroMagnetic.LLG
        check(ccall((:mm_set_llg, libmmcuda), Cint, (Ptr{Cvoid}, Float64, Float64, Cint),
                    h.ptr, drv.alpha, drv.gamma, drv.precession ? 1 : 0))
        if drv.integrator isa MicroMagnetic.AdaptiveRK
            # method of Sim(mesh; integrator=...)  src/integrator/adaptive_rk.jl:248-266
            meth = drv.integrator.method
            code = meth isa MicroMagnetic.BS23Method ? 1 : meth isa MicroMagnetic.CashKarp54Method ? 2 :
                   meth isa MicroMagnetic.Fehlberg54Method ? 3 : 0
            check(ccall((:mm_set_adaptive_method, libmmcuda), Cint, (Ptr{Cvoid}, Cint), h.ptr, code))
            check(ccall((:mm_dopri_set_tol, libmmcuda), Cint, (Ptr{Cvoid}, Float64), h.ptr, drv.integrator.tol))
        end
    end
    for term in sim.interactions
        add_term!(h, term)
    end
    HANDLES[sim] = h
    return h
end

add_term!(h, z::MicroMagnetic.Zeeman) =
    check(ccall((:mm_add_zeeman, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}, Float64, Float64, Float64),
                h.ptr, f64(z.field), 0.0, 0.0, 0.0))
add_term!(h, e::MicroMagnetic.UniformExchange) =
    check(ccall((:mm_add_exch, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}, Float64, Float64, Float64),
                h.ptr, C_NULL, e.Ax, e.Ay, e.Az))
add_term!(h, e::MicroMagnetic.SpatialExchange) =
    check(ccall((:mm_add_exch, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}, Float64, Float64, Float64),
                h.ptr, f64(e.A), 0.0, 0.0, 0.0))
add_term!(h, d::MicroMagnetic.BulkDMI) =
    check(ccall((:mm_add_dmi_bulk, libmmcuda), Cint, (Ptr{Cvoid}, Float64, Float64, Float64), h.ptr, d.Dx, d.Dy, d.Dz))
add_term!(h, d::MicroMagnetic.InterfacialDMI) =
    check(ccall((:mm_add_dmi_interfacial, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}, Float64), h.ptr, f64(d.D), 0.0))
add_term!(h, a::MicroMagnetic.Anisotropy) =
    check(ccall((:mm_add_anis, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}, Float64, Float64, Float64, Float64),
                h.ptr, f64(a.Ku), 0.0, a.axis[1], a.axis[2], a.axis[3]))
# Demag: the Newell tensor with macro-PBC images is re-assembled on the device
add_term!(h, d::MicroMagnetic.Demag) =
    check(ccall((:mm_add_demag, libmmcuda), Cint, (Ptr{Cvoid}, Cint, Cint, Cint), h.ptr, 0, 0, 0))
add_term!(h, t) = error("term $(typeof(t)) is not on the accelerated path")

handle(sim) = get(HANDLES, sim, nothing)

# sim.spin crosses the boundary in its own element type: Float32 in the
# reference's Float32 mode (set_precision(Float32), src/MicroMagnetic.jl:22-38)
function push_spin!(h, spin)
    a = Array(spin)
    if eltype(a) == Float32
        check(ccall((:mm_set_m_f32, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float32}), h.ptr, Vector{Float32}(a)))
    else
        check(ccall((:mm_set_m, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}), h.ptr, f64(a)))
    end
    return nothing
end

function pull_spin!(sim, h)
    if eltype(sim.spin) == Float32
        m = Vector{Float32}(undef, 3 * h.n)
        check(ccall((:mm_get_m_f32, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float32}), h.ptr, m))
    else
        m = Vector{Float64}(undef, 3 * h.n)
        check(ccall((:mm_get_m, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}), h.ptr, m))
    end
    copyto!(sim.spin, m)
    return sim.spin
end

# effective_field(sim, spin, t)  src/micro/field.jl:496-505
function effective_field(sim::MicroMagnetic.MicroSim, spin, t::Float64=0.0)
    h = handle(sim)
    h === nothing && return invoke(effective_field, Tuple{MicroMagnetic.AbstractSim,Any,Float64}, sim, spin, t)
    push_spin!(h, spin)
    H = Vector{Float64}(undef, 3 * h.n)
    check(ccall((:mm_effective_field, libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}), h.ptr, H))
    copyto!(sim.field, H)
    return nothing
end

# advance_step(sim, ::RungeKutta)  src/integrator/rk.jl:23-52
function advance_step(sim::MicroMagnetic.MicroSim, integ::MicroMagnetic.RungeKutta)
    h = handle(sim)
    h === nothing && return invoke(advance_step, Tuple{MicroMagnetic.AbstractSim,MicroMagnetic.RungeKutta}, sim, integ)
    check(ccall((:mm_rk4_run, libmmcuda), Cint, (Ptr{Cvoid}, Float64, Int64), h.ptr, integ.step, 1))
    integ.nsteps += 1
    integ.t = integ.nsteps * integ.step
    pull_spin!(sim, h)
    return nothing
end

# advance_step(sim, ::ModifiedEuler)  src/integrator/heun.jl:28-49
function advance_step(sim::MicroMagnetic.MicroSim, integ::MicroMagnetic.ModifiedEuler)
    h = handle(sim)
    h === nothing && return invoke(advance_step, Tuple{MicroMagnetic.AbstractSim,MicroMagnetic.ModifiedEuler}, sim, integ)
    check(ccall((:mm_heun_run, libmmcuda), Cint, (Ptr{Cvoid}, Float64, Int64), h.ptr, integ.step, 1))
    integ.nsteps += 1
    integ.t = integ.nsteps * integ.step
    pull_spin!(sim, h)
    return nothing
end

# save_ovf(sim, fname; type) from the device state  src/ovf2.jl:44-62
function save_ovf(sim::MicroMagnetic.MicroSim, fname::String; type::DataType=Float64)
    h = handle(sim)
    h === nothing && return MicroMagnetic.save_ovf(sim, fname; type=type)
    code = type == Float32 ? 4 : type == String ? 0 : 8
    check(ccall((:mm_save_ovf, libmmcuda), Cint, (Ptr{Cvoid}, Cstring, Cint, Cstring), h.ptr, fname, code, sim.name))
    return nothing
end

# run_until(sim, t_end) with Dormand-Prince  src/sim.jl:547-574
function run_until(sim::MicroMagnetic.MicroSim, t_end::Float64, integ::MicroMagnetic.AdaptiveRK, save_data::Bool)
    h = handle(sim)
    h === nothing && return invoke(run_until, Tuple{MicroMagnetic.AbstractSim,Float64,MicroMagnetic.Integrator,Bool},
                                   sim, t_end, integ, save_data)
    st = Ref(Stats())
    check(ccall((:mm_run_until, libmmcuda), Cint, (Ptr{Cvoid}, Float64, Ref{Stats}), h.ptr, t_end, st))
    integ.t, integ.step, integ.step_next = st[].t, st[].step, st[].step_next
    integ.nsteps, integ.nfevals = st[].nsteps, st[].nfevals
    pull_spin!(sim, h)
    sim.saver.t = t_end
    if save_data
        compute_system_energy(sim, sim.spin, t_end)
        MicroMagnetic.write_data(sim)
    end
    sim.saver.nsteps += 1
    return nothing
end

# relax(sim; max_steps, stopping_dmdt)  src/sim.jl:392-490
function relax(sim::MicroMagnetic.MicroSim; max_steps=10000, stopping_dmdt=0.01, kwargs...)
    h = handle(sim)
    h === nothing && return invoke(relax, Tuple{MicroMagnetic.AbstractSim}, sim; max_steps=max_steps,
                                   stopping_dmdt=stopping_dmdt, kwargs...)
    drv = sim.driver isa MicroMagnetic.SD ? 0 : 1
    steps = Ref{Int64}(0); mx = Ref{Float64}(0)
    check(ccall((:mm_relax, libmmcuda), Cint, (Ptr{Cvoid}, Cint, Int64, Float64, Ref{Int64}, Ref{Float64}),
                h.ptr, drv, max_steps, stopping_dmdt, steps, mx))
    pull_spin!(sim, h)
    return nothing
end

# compute_system_energy  src/micro/field.jl:520-536 (FP64 device reductions)
function compute_system_energy(sim::MicroMagnetic.MicroSim, spin, t::Float64)
    h = handle(sim)
    h === nothing && return invoke(compute_system_energy, Tuple{MicroMagnetic.AbstractSim,AbstractArray,Float64}, sim, spin, t)
    for term in sim.interactions
        hasproperty(term, :energy) || continue
        k = term_index(term)
        k < 0 && continue
        e = Vector{Float64}(undef, h.n)
        check(ccall((:mm_term_field, libmmcuda), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}),
                    h.ptr, k, C_NULL, e))
        copyto!(term.energy, e)
    end
    return 0
end

term_index(::MicroMagnetic.Zeeman) = 0
term_index(::Union{MicroMagnetic.UniformExchange,MicroMagnetic.SpatialExchange}) = 1
term_index(::MicroMagnetic.BulkDMI) = 2
term_index(::MicroMagnetic.InterfacialDMI) = 3
term_index(::MicroMagnetic.Anisotropy) = 4
term_index(::MicroMagnetic.Demag) = 5
term_index(_) = -1

end # module
