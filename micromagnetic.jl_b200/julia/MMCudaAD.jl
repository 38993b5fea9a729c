# MMCudaAD.jl -- reverse-mode rule for fixed-step RK4 on the device.
#
# The reference has no differentiation of the LLG path.  This file gives a
# ChainRulesCore.rrule for `rk4_final(sim, m0, nsteps)` (m after nsteps RK4
# steps of advance_step(sim, ::RungeKutta), src/integrator/rk.jl:23-52) whose
# pullback is libmmcuda's discrete adjoint (mm_adjoint_record /
# mm_adjoint_backward): dL/dm0, and the parameter gradients dL/dMs (per cell,
# A/m), dL/dKu and dL/dD (interfacial DMI, per cell) left in
# `MMCuda.ADJOINT_GRADS[sim]`.  Include after MMCuda.jl, with ChainRulesCore
# in the environment:
#
#     using ChainRulesCore, Zygote
#     include("MMCuda.jl"); include("MMCudaAD.jl"); using .MMCuda
#     MMCuda.attach!(sim)
#     loss(m0) = sum(abs2, MMCuda.rk4_final(sim, m0, 2000) .- target)
#     g = Zygote.gradient(loss, m0)[1]
using ChainRulesCore

const ADJOINT_GRADS = IdDict{Any,Dict{Symbol,Vector{Float64}}}()

function rk4_final(sim::MicroMagnetic.MicroSim, m0::AbstractVector, nsteps::Integer; ckpt_every::Integer=100)
    h = MMCuda.handle(sim)
    MMCuda.check(ccall((:mm_set_m, MMCuda.libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}), h.ptr, Float64.(m0)))
    MMCuda.check(ccall((:mm_rk4_run, MMCuda.libmmcuda), Cint, (Ptr{Cvoid}, Float64, Int64), h.ptr,
                       sim.driver.integrator.step, nsteps))
    m = Vector{Float64}(undef, 3 * h.n)
    MMCuda.check(ccall((:mm_get_m, MMCuda.libmmcuda), Cint, (Ptr{Cvoid}, Ptr{Float64}), h.ptr, m))
    return m
end

function ChainRulesCore.rrule(::typeof(rk4_final), sim::MicroMagnetic.MicroSim, m0::AbstractVector,
                              nsteps::Integer; ckpt_every::Integer=100)
    h = MMCuda.handle(sim)
    lib = MMCuda.libmmcuda
    MMCuda.check(ccall((:mm_set_m, lib), Cint, (Ptr{Cvoid}, Ptr{Float64}), h.ptr, Float64.(m0)))
    MMCuda.check(ccall((:mm_adjoint_record, lib), Cint, (Ptr{Cvoid}, Float64, Int64, Int64), h.ptr,
                       sim.driver.integrator.step, nsteps, ckpt_every))
    mT = Vector{Float64}(undef, 3 * h.n)
    MMCuda.check(ccall((:mm_get_m, lib), Cint, (Ptr{Cvoid}, Ptr{Float64}), h.ptr, mT))
    function rk4_final_pullback(ΔmT)
        n = h.n
        gm0, gMs, gKu, gD = zeros(3n), zeros(n), zeros(n), zeros(n)
        MMCuda.check(ccall((:mm_adjoint_backward, lib), Cint,
                           (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                           h.ptr, Float64.(unthunk(ΔmT)), gm0, gMs, gKu, gD))
        ADJOINT_GRADS[sim] = Dict(:Ms => gMs, :Ku => gKu, :D => gD)
        return NoTangent(), NoTangent(), gm0, NoTangent()
    end
    return mT, rk4_final_pullback
end
