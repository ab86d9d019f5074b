"""
    DoNOFB200

Julia side of libdonofb200, the B200 (sm_100a) library of DoNOF.jl's RI hot
path.  Every function here is one `ccall` into the C ABI declared in
`include/donof_b200.h`; the arrays pass through unchanged (FP64,
column-major: Julia's own layout).  DoNOF.jl reaches these functions through
its GPU package extension `DoNOFGPUExt` (julia/ext/DoNOFGPUExt.jl), selected
by `using DoNOF, DoNOFB200`.

The library is found at `ENV["DONOF_B200_LIB"]` when that is set at
precompile time, else at its in-tree build location.
"""
module DoNOFB200

export B200Tensor

const libdonof = get(ENV, "DONOF_B200_LIB",
                     normpath(joinpath(@__DIR__, "..", "..", "..", "donof.jl_b200", "donof_b200",
                                       "libdonofb200.so")))

const DONOF_OK = Cint(0)
const PREC_FP64 = Cint(0)
const PREC_MIXED = Cint(1)
const ORB_METHODS = Dict("ADAM" => Cint(0), "ADABelief" => Cint(1), "YOGI" => Cint(2), "Demon" => Cint(3))

# ---------------------------------------------------------------- context and errors
const CTX = Ref{Ptr{Cvoid}}(C_NULL)

"""Text of the last failure on `ctx` (or of a call made before any context existed)."""
last_error(ctx::Ptr{Cvoid} = CTX[]) =
    unsafe_string(ccall((:donof_last_error, libdonof), Cstring, (Ptr{Cvoid},), ctx))

"""Raises a Julia error for a non-zero status, as DoNOF.jl's own code raises exceptions."""
function check(status::Cint, ctx::Ptr{Cvoid} = CTX[])
    status == DONOF_OK && return nothing
    error("libdonofb200 status $(status): $(last_error(ctx))")
end

"""The process's library context on device 0 (its own CUDA stream), created on first use."""
function context()
    if CTX[] == C_NULL
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:donof_create, libdonof), Cint, (Cint, Ref{Ptr{Cvoid}}), Cint(0), r), C_NULL)
        CTX[] = r[]
    end
    return CTX[]
end

"""Failures the context's kernels recorded since the last read (bit mask), cleared by the read."""
function error_flags()
    f = Ref{Cint}(0)
    check(ccall((:donof_error_flags, libdonof), Cint, (Ptr{Cvoid}, Ref{Cint}), context(), f))
    return Int(f[])
end

dense(x::Array{Float64}) = x
dense(x) = Array{Float64}(x)

# ---------------------------------------------------------------- the RI tensor
"""
    B200Tensor

The RI tensor b[m, n, l] resident on the GPU (a library job).  It stands
where DoNOF.jl's extension keeps a `CuArray{Float64,3}`: `size` works, and the
hot functions of DoNOF.jl dispatch on it.
"""
mutable struct B200Tensor <: AbstractArray{Float64,3}
    job::Ptr{Cvoid}
    nbf::Int
    naux::Int
    function B200Tensor(job::Ptr{Cvoid}, nbf::Integer, naux::Integer)
        b = new(job, Int(nbf), Int(naux))
        finalizer(free!, b)
        return b
    end
end
Base.size(b::B200Tensor) = (b.nbf, b.nbf, b.naux)
Base.getindex(::B200Tensor, ::Int...) = error("a B200Tensor lives on the GPU: use the library calls")

function free!(b::B200Tensor)
    if b.job != C_NULL
        ccall((:donof_job_free, libdonof), Cint, (Ptr{Cvoid},), b.job)
        b.job = C_NULL
    end
    return nothing
end

"""Copies b to the device (eris_to_gpu); `precision = PREC_MIXED` also keeps its bf16 split."""
function upload(I::Array{Float64,3}; precision::Integer = PREC_FP64)
    nbf, nbf2, naux = size(I)
    nbf == nbf2 || throw(DimensionMismatch("b must be nbf x nbf x naux"))
    job = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:donof_b_upload, libdonof), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Cint, Cint, Cint, Ref{Ptr{Cvoid}}),
                context(), I, nbf, naux, precision, job))
    return B200Tensor(job[], nbf, naux)
end

"""b = I G^{-1/2} built on the device (Iaux / Iaux_gpu followed by eris_to_gpu)."""
function iaux(G::Matrix{Float64}, I::Array{Float64,3}; precision::Integer = PREC_FP64)
    nbf, _, naux = size(I)
    size(G) == (naux, naux) || throw(DimensionMismatch("G must be naux x naux"))
    job = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:donof_iaux, libdonof), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Cint, Cint, Cint, Ref{Ptr{Cvoid}}),
                context(), G, I, nbf, naux, precision, job))
    return B200Tensor(job[], nbf, naux)
end

"""Form used by later calls on b: PREC_FP64, or PREC_MIXED for a tensor uploaded with it."""
set_precision!(b::B200Tensor, precision::Integer) =
    check(ccall((:donof_job_set_precision, libdonof), Cint, (Ptr{Cvoid}, Cint), b.job, precision))

"""FP64 form: run the first contraction (b_l C5) on the tensor cores from int8 digit
slices of b (exact integer products, within ~1e-13 of the FP64 GEMM), or back on the
FP64 GEMM with `enable = false`."""
set_fp64_tc!(b::B200Tensor, enable::Bool=true) =
    check(ccall((:donof_job_set_fp64_tc, libdonof), Cint, (Ptr{Cvoid}, Cint), b.job, enable ? 1 : 0))

# ---------------------------------------------------------------- the hot path
"""compute_Lagrange2 (src/utils.jl:1-59): (elag, H_mat, E_elec)."""
function lagrange2(C, n, H, b::B200Tensor, cj12, ck12, nalpha, nbeta)
    nbf5 = length(n)
    elag = zeros(b.nbf, b.nbf)
    H_mat = zeros(b.nbf, nbf5)
    E = Ref{Float64}(0.0)
    check(ccall((:donof_lagrange2, libdonof), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                 Cint, Cint, Cint, Ptr{Float64}, Ptr{Float64}, Ref{Float64}),
                b.job, dense(C), dense(n), dense(H), dense(cj12), dense(ck12), nbf5, nalpha, nbeta,
                elag, H_mat, E))
    return elag, H_mat, E[]
end

"""JKH_MO (src/integrals.jl:144-172): (J_MO, K_MO, H_core)."""
function jkh_mo(C, H, b::B200Tensor, nbf5::Integer)
    J = zeros(nbf5, nbf5)
    K = zeros(nbf5, nbf5)
    Hc = zeros(nbf5)
    check(ccall((:donof_jkh_mo, libdonof), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                b.job, dense(C), dense(H), nbf5, J, K, Hc))
    return J, K, Hc
end

"""rotate_orbital (src/utils.jl:499-521), in FP64: C exp(Y(y))."""
function rotate(y, C, nbf::Integer, nbf5::Integer)
    Cnew = zeros(nbf, nbf)
    check(ccall((:donof_rotate, libdonof), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Cint, Cint, Ptr{Float64}, Ptr{Float64}),
                context(), dense(y), nbf, nbf5, dense(C), Cnew))
    return Cnew
end

"""calcorbg (src/pnof.jl:1389-1407): the packed orbital gradient at y."""
function orbgrad(y, n, cj12, ck12, C, H, b::B200Tensor, nalpha, nbeta)
    nbf5 = length(n)
    nvar = nbf5 * b.nbf - div(nbf5 * (nbf5 + 1), 2)
    grad = zeros(nvar)
    check(ccall((:donof_orbgrad, libdonof), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                 Ptr{Float64}, Cint, Cint, Cint, Ptr{Float64}),
                b.job, dense(y), dense(C), dense(n), dense(H), dense(cj12), dense(ck12), nbf5, nalpha,
                nbeta, grad))
    return grad
end

"""
The host side of one iteration of the optimiser loop (src/minimization.jl:390-412)
for a caller that drives it through `rotate` and `lagrange2`: packs calcorbg's
gradient from `elag` into `g` and updates `m`, `v`, `vmax` and `y` in place
(donof_orb_step_host, compiled code).  Returns max|g|.
"""
function orb_step_host!(method::AbstractString, it::Integer, maxloop::Integer, alpha::Real,
                        elag::Matrix{Float64}, nbf5::Integer, g, m, v, vmax, y)
    gmax = Ref{Float64}(0.0)
    check(ccall((:donof_orb_step_host, libdonof), Cint,
                (Cint, Cint, Cint, Cdouble, Ptr{Float64}, Cint, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                 Ptr{Float64}, Ptr{Float64}, Ref{Float64}),
                ORB_METHODS[method], it, maxloop, alpha, elag, size(elag, 1), nbf5, g, m, v, vmax, y, gmax),
          Ptr{Cvoid}(C_NULL))
    return gmax[]
end

# --- integral front end (in place of GaussianBasis.jl in compute_integrals,
# src/integrals.jl:1-49): shells as flat arrays (l, centre in bohr, primitive
# counts, exponents, contraction coefficients as a basis-set file prints them).
mutable struct B200Basis
    handle::Ptr{Cvoid}
    nbas::Int
end

function basis(l::Vector{Cint}, centre::Vector{Float64}, nprim::Vector{Cint}, exps::Vector{Float64},
               coefs::Vector{Float64}; spherical::Bool = true)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:donof_basis_create, libdonof), Cint,
                (Cint, Ptr{Cint}, Ptr{Float64}, Ptr{Cint}, Ptr{Float64}, Ptr{Float64}, Cint, Ref{Ptr{Cvoid}}),
                length(l), l, centre, nprim, exps, coefs, spherical, h), Ptr{Cvoid}(C_NULL))
    nb = ccall((:donof_basis_nbf, libdonof), Cint, (Ptr{Cvoid},), h[])
    bs = B200Basis(h[], nb)
    finalizer(x -> ccall((:donof_basis_free, libdonof), Cint, (Ptr{Cvoid},), x.handle), bs)
    return bs
end

"""S, T, V (overlap, kinetic, nuclear with the nuclei Z at xyz, bohr, 3 x natom)."""
function int1e(b::B200Basis, Z::Vector{Float64}, xyz::Matrix{Float64})
    S, T, V = zeros(b.nbas, b.nbas), zeros(b.nbas, b.nbas), zeros(b.nbas, b.nbas)
    check(ccall((:donof_int1e, libdonof), Cint,
                (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                b.handle, length(Z), Z, xyz, S, T, V), Ptr{Cvoid}(C_NULL))
    return S, T, V
end

"""ERI_2e2c: G[P, Q] = (P|Q) over the auxiliary basis."""
function int2c2e(aux::B200Basis)
    G = zeros(aux.nbas, aux.nbas)
    check(ccall((:donof_int2c2e, libdonof), Cint, (Ptr{Cvoid}, Ptr{Float64}), aux.handle, G), Ptr{Cvoid}(C_NULL))
    return G
end

"""ERI_2e3c: I[m, n, P] = (mn|P) (host threads); `iaux(int2c2e(aux), int3c2e(b, aux))` then gives the job's b."""
function int3c2e(b::B200Basis, aux::B200Basis)
    I = zeros(b.nbas, b.nbas, aux.nbas)
    check(ccall((:donof_int3c2e, libdonof), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}),
                b.handle, aux.handle, I), Ptr{Cvoid}(C_NULL))
    return I
end

"""
One orbopt_adam / _adabelief / _yogi / _demon call (src/minimization.jl:242-630)
with the whole loop on the device.  `alpha` and `maxloop` are read and updated
like p.alpha and p.maxloop.  Returns (E, C, nit, success).
"""
function orbopt(method::AbstractString, n, cj12, ck12, H, C, b::B200Tensor, nalpha, nbeta,
                alpha::Ref{Float64}, maxloop::Ref{Cint}, threshgorb::Real)
    Cio = copy(dense(C))
    E = Ref{Float64}(0.0)
    nit = Ref{Cint}(0)
    ok = Ref{Cint}(0)
    check(ccall((:donof_orbopt, libdonof), Cint,
                (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Cint, Cint, Cint,
                 Ref{Float64}, Ref{Cint}, Cdouble, Ptr{Float64}, Ref{Float64}, Ref{Cint}, Ref{Cint}),
                b.job, ORB_METHODS[method], dense(n), dense(cj12), dense(ck12), dense(H), length(n), nalpha,
                nbeta, alpha, maxloop, threshgorb, Cio, E, nit, ok))
    return E[], Cio, Int(nit[]), ok[] != 0
end

# ---------------------------------------------------------------- the energy loop
struct OccParams
    nbf5::Cint
    no1::Cint
    nbeta::Cint
    nalpha::Cint
    ncwo::Cint
    ista::Cint
    high_spin::Cint
    occ_method::Cint
    h_cut::Cdouble
end

struct EnergyParams
    occ::OccParams
    orb_method::Cint
    maxit::Cint
    maxloop::Cint
    alpha::Cdouble
    threshgorb::Cdouble
    threshgocc::Cdouble
    threshen::Cdouble
    order_subspaces::Cint
    freeze_occ::Cint
    stop_rel_de::Cdouble
    occ_device::Cint
end

struct EnergyResult
    E_elec::Cdouble
    iterations::Cint
    converged::Cint
    tot_it_orb::Cint
    tot_it_occ::Cint
    max_grad_orb::Cdouble
    norm_grad_occ::Cdouble
end

"""EnergyParams of DoNOF's Param `p` (the names of src/param.jl)."""
energy_params(p; freeze_occ::Bool = false, stop_rel_de::Real = 0.0, occ_device::Bool = false) =
    EnergyParams(OccParams(p.nbf5, p.no1, p.nbeta, p.nalpha, p.ncwo, p.ista, p.HighSpin,
                           p.occ_method == "Softmax" ? 0 : 1, p.h_cut),
                 ORB_METHODS[p.orb_method], p.maxit, p.maxloop, p.alpha, p.threshgorb, p.threshgocc,
                 p.threshen, p.ipnof > 4, freeze_occ, stop_rel_de, occ_device)

"""
The orbital / occupation alternation of DoNOF.energy (src/energy.jl:140-224)
in one call, in b's precision.  C and gamma are updated in place; p.alpha and
p.maxloop carry the optimiser's state back.  Returns (E_elec, n, elag, result).
"""
function energy_loop!(b::B200Tensor, p, H, C::Matrix{Float64}, gamma::Vector{Float64}; freeze_occ::Bool = false,
                      stop_rel_de::Real = 0.0)
    prm = Ref(energy_params(p; freeze_occ = freeze_occ, stop_rel_de = stop_rel_de))
    res = Ref{EnergyResult}()
    n = zeros(p.nbf5)
    elag = zeros(b.nbf, b.nbf)
    check(ccall((:donof_energy, libdonof), Cint,
                (Ptr{Cvoid}, Ref{EnergyParams}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                 Ptr{Float64}, Ptr{Float64}, Ref{EnergyResult}),
                b.job, prm, dense(H), C, gamma, n, elag, C_NULL, res))
    p.alpha = prm[].alpha
    p.maxloop = prm[].maxloop
    return res[].E_elec, n, elag, res[]
end

end # module
