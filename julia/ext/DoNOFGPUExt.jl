# DoNOF.jl's GPU package extension, backed by libdonofb200 (B200, sm_100a).
#
# This file replaces DoNOF.jl's ext/DoNOFGPUExt.jl and keeps its module name,
# so that compute_integrals (src/integrals.jl:50-62) finds it with
# Base.get_extension(@__MODULE__, :DoNOFGPUExt) and routes the RI tensor
# through Iaux_gpu / eris_to_gpu below.  DoNOF.jl's Project.toml selects it
# with the entries of julia/DoNOF.Project.extensions.toml
# ([weakdeps] DoNOFB200, [extensions] DoNOFGPUExt = "DoNOFB200"); a session
# activates it with `using DoNOF, DoNOFB200`.
#
# I becomes a DoNOFB200.B200Tensor, and the methods below are then picked by
# dispatch wherever DoNOF.energy(bset, p) calls the hot path:
#   Iaux_gpu, eris_to_gpu        ext/DoNOFGPUExt.jl:9-50
#   computeJKH_MO, JKH_MO        ext/DoNOFGPUExt.jl:52-94  (src/integrals.jl:131-172)
#   compute_Lagrange2            ext/DoNOFGPUExt.jl:150-245 (src/utils.jl:1-59)
#   rotate_orbital               ext/DoNOFGPUExt.jl:355-382 (src/utils.jl:499-521), FP64 here
#   calcorbg                     src/pnof.jl:1389-1407
#   orbopt_adam / _adabelief /   src/minimization.jl:242-630, each one library call
#   _yogi / _demon               with the whole loop on the device
# ENERGY1r, occoptr and the energy loop itself stay DoNOF.jl's: they reach the
# library through compute_Lagrange2 and computeJKH_MO.
module DoNOFGPUExt

using DoNOF
using DoNOFB200
using DoNOFB200: B200Tensor

# precision of the uploaded tensor: FP64 unless DONOF_B200_PRECISION=mixed
# (the mixed form also keeps a bf16 split; set_precision! switches between them)
upload_precision() = get(ENV, "DONOF_B200_PRECISION", "fp64") == "mixed" ? DoNOFB200.PREC_MIXED :
                     DoNOFB200.PREC_FP64

# ---- integrals hook (src/integrals.jl:50-62)
Iaux_gpu(G::Matrix{Float64}, I::Array{Float64,3}) = DoNOFB200.iaux(G, I; precision = upload_precision())

eris_to_gpu(I::Array{Float64,3}) = DoNOFB200.upload(I; precision = upload_precision())
eris_to_gpu(I::B200Tensor) = I                 # already on the device (after Iaux_gpu)
eris_to_gpu(I::Array{Float64,4}) = I           # 4-index ERIs (p.RI = false) stay on DoNOF.jl's CPU path

# ---- JKH_MO, RI method
DoNOF.computeJKH_MO(C, H, I::B200Tensor, p) = DoNOF.JKH_MO(C, H, I, p.nbf, p.nbf5, p.nbfaux)
DoNOF.JKH_MO(C, H, b::B200Tensor, nbf, nbf5, nbfaux) = DoNOFB200.jkh_mo(C, H, b, nbf5)

# ---- compute_Lagrange2, RI method
function DoNOF.compute_Lagrange2(C, n, H, b::B200Tensor, cj12, ck12, nalpha, nbeta)
    elag, H_mat, _ = DoNOFB200.lagrange2(C, n, H, b, cj12, ck12, nalpha, nbeta)
    return elag, H_mat
end

# ---- rotate_orbital (the CUDA.jl extension also takes over y::Array)
DoNOF.rotate_orbital(y::Array, C, p) = DoNOFB200.rotate(y, C, p.nbf, p.nbf5)

# ---- calcorbg
DoNOF.calcorbg(y, n, cj12, ck12, C, H, I::B200Tensor, pa) =
    DoNOFB200.orbgrad(y, n, cj12, ck12, C, H, I, pa.nalpha, pa.nbeta)

# ---- the ADAM-family orbital optimisers, one device-resident loop per call
function device_orbopt(method, gamma, C, H, I::B200Tensor, p)
    n, _ = DoNOF.ocupacion(gamma, p.no1, p.ndoc, p.nalpha, p.nv, p.nbf5, p.ndns, p.ncwo, p.HighSpin,
                           p.occ_method)
    cj12, ck12 = DoNOF.PNOFi_selector(n, p)
    alpha = Ref{Float64}(p.alpha)
    maxloop = Ref{Cint}(p.maxloop)
    E, Cnew, nit, success = DoNOFB200.orbopt(method, n, cj12, ck12, H, C, I, p.nalpha, p.nbeta, alpha, maxloop,
                                             p.threshgorb)
    p.alpha = alpha[]
    p.maxloop = maxloop[]
    return E, Cnew, nit, success
end

DoNOF.orbopt_adam(gamma, C, H, I::B200Tensor, p) = device_orbopt("ADAM", gamma, C, H, I, p)
DoNOF.orbopt_adabelief(gamma, C, H, I::B200Tensor, p) = device_orbopt("ADABelief", gamma, C, H, I, p)
DoNOF.orbopt_yogi(gamma, C, H, I::B200Tensor, p) = device_orbopt("YOGI", gamma, C, H, I, p)
DoNOF.orbopt_demon(gamma, C, H, I::B200Tensor, p) = device_orbopt("Demon", gamma, C, H, I, p)

end # module
