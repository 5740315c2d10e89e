# CutAndDisplaceB200 — Julia bindings of libcad_td.so (the B200 TD path).
#
# Drop-in methods for CutAndDisplaceJulia's TD (its three overloads), TD_sum,
# CalculateInfluenceMatrices3D and the plain SlipCalculator3D: same names,
# argument order and meaning, the parent module's result types (StrainInf,
# DispInf, Strains, Disps, TractionInf) and boundary-condition types, same
# error texts.  Each method checks dimensions as the reference does, then
# ccalls the C ABI declared in include/cad_td.h.  Include it inside
# CutAndDisplaceJulia (its parent module supplies the types and
# SetupTractionVector), then call these methods in place of the reference's:
#
#     include("CutAndDisplaceB200.jl"); using .CutAndDisplaceB200
#     CutAndDisplaceB200.TD(X, Y, Z, P1, P2, P3, Dss, Dds, Dn, ν, G, 1, 1, 0)
module CutAndDisplaceB200

const libcad = get(ENV, "CAD_TD_LIB", joinpath(@__DIR__, "..", "libcad_td.so"))
# the module this file is included into: CutAndDisplaceJulia, whose struct
# types the methods below take and return
const Ref_ = parentmodule(@__MODULE__)

const _ctx = Ref{Ptr{Cvoid}}(C_NULL)

function ctx()
    if _ctx[] == C_NULL
        h = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:cad_init, libcad), Cint, (Cint, Ref{Ptr{Cvoid}}), 0, h)
        rc == 0 || error("cad_init failed (status $rc): a CUDA device is required")
        _ctx[] = h[]
    end
    return _ctx[]
end

function check(rc)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:cad_last_error, libcad), Cstring, (Ptr{Cvoid},), ctx()))
    error(msg)
end

f64(a) = convert(Array{Float64}, a)

function dims_ok(P1, P2, P3, Dss, Dds, Dn)
    n = size(P1, 1); if length(P1) == 3; n = 1; end
    n == size(P2, 1) && n == size(P3, 1) && n == length(Dds) && n == length(Dss) && n == length(Dn)
end

const _td_sig = (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Ptr{Float64}, Ptr{Float64},
                 Ptr{Float64}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Cint, Cint, Cint,
                 Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}})

# TD, influence-matrix fill overload (src/TD.jl:135): fills the caller's
# StrainInf / DispInf matrices (M x N, as the reference preallocates them)
function TD(X, Y, Z, P1List, P2List, P3List, Dss, Dds, Dn, ν, G, DispFlag, StrainFlag, HSflag,
            StrainInfMat::Ref_.StrainInf, DispInfMat::Ref_.DispInf)
    dims_ok(P1List, P2List, P3List, Dss, Dds, Dn) || error("Element size inputs must be the same dimensions")
    M = length(X); N = length(P1List) == 3 ? 1 : size(P1List, 1)
    S = StrainFlag == 1 ? [getfield(StrainInfMat, k) for k in 1:18] : Matrix{Float64}[]
    U = DispFlag == 1 ? [getfield(DispInfMat, k) for k in 1:9] : Matrix{Float64}[]
    all(a -> a isa Matrix{Float64} && size(a) == (M, N), vcat(S, U)) ||
        error("Element size inputs must be the same dimensions")
    sp = [pointer(a) for a in S]; up = [pointer(a) for a in U]
    GC.@preserve S U sp up begin
        check(ccall((:cad_td_inf, libcad), Cint, _td_sig,
            ctx(), f64(vec(X)), f64(vec(Y)), f64(vec(Z)), M, f64(P1List), f64(P2List), f64(P3List), N,
            f64(vec(Dss)), f64(vec(Dds)), f64(vec(Dn)), ν, G, DispFlag, StrainFlag, HSflag,
            StrainFlag == 1 ? sp : C_NULL, DispFlag == 1 ? up : C_NULL))
    end
    return (StrainInfMat, DispInfMat)
end

# TD, allocating overload (src/TD.jl:77): zeros of the flagged fields, then the fill
function TD(X, Y, Z, P1List, P2List, P3List, Dss, Dds, Dn, ν, G, DispFlag, StrainFlag, HSflag)
    M = length(X); N = length(P1List) == 3 ? 1 : size(P1List, 1)
    S = StrainFlag == 1 ? Ref_.StrainInf((zeros(M, N) for _ in 1:18)...) : Ref_.StrainInf(([] for _ in 1:18)...)
    U = DispFlag == 1 ? Ref_.DispInf((zeros(M, N) for _ in 1:9)...) : Ref_.DispInf(([] for _ in 1:9)...)
    return TD(X, Y, Z, P1List, P2List, P3List, Dss, Dds, Dn, ν, G, DispFlag, StrainFlag, HSflag, S, U)
end

# TD, summing overload (src/TD.jl:219): Strains / Disps summed over triangles
# and modes, reshaped like X (the arguments only select this overload)
function TD(X, Y, Z, P1List, P2List, P3List, Dss, Dds, Dn, ν, G, DispFlag, StrainFlag, HSflag,
            StrainInfVector::Ref_.Strains, DispInfVector::Ref_.Disps)
    dims_ok(P1List, P2List, P3List, Dss, Dds, Dn) || error("Element size inputs must be the same dimensions")
    M = length(X); N = length(P1List) == 3 ? 1 : size(P1List, 1)
    S = [zeros(M) for _ in 1:6]; U = [zeros(M) for _ in 1:3]
    sp = [pointer(a) for a in S]; up = [pointer(a) for a in U]
    GC.@preserve S U sp up begin
        check(ccall((:cad_td_sum_eval, libcad), Cint, _td_sig,
            ctx(), f64(vec(X)), f64(vec(Y)), f64(vec(Z)), M, f64(P1List), f64(P2List), f64(P3List), N,
            f64(vec(Dss)), f64(vec(Dds)), f64(vec(Dn)), ν, G, DispFlag, StrainFlag, HSflag, sp, up))
    end
    shape(a) = size(X, 2) != 1 ? reshape(a, size(X)) : a
    Sv = StrainFlag == 1 ? Ref_.Strains((shape(a) for a in S)...) : Ref_.Strains([], [], [], [], [], [])
    Uv = DispFlag == 1 ? Ref_.Disps((shape(a) for a in U)...) : Ref_.Disps([], [], [])
    return (Sv, Uv)
end

# TD_sum: 18 strain + 9 displacement M x N matrices -> nine M x 1 sums (empty in, empty out)
function TD_sum(ExxDn, EyyDn, EzzDn, ExyDn, ExzDn, EyzDn, ExxDss, EyyDss, EzzDss, ExyDss, ExzDss, EyzDss,
                ExxDds, EyyDds, EzzDds, ExyDds, ExzDds, EyzDds, UxDn, UyDn, UzDn, UxDss, UyDss, UzDss,
                UxDds, UyDds, UzDds)
    Sin = [ExxDn, EyyDn, EzzDn, ExyDn, ExzDn, EyzDn, ExxDss, EyyDss, EzzDss, ExyDss, ExzDss, EyzDss,
           ExxDds, EyyDds, EzzDds, ExyDds, ExzDds, EyzDds]
    Uin = [UxDn, UyDn, UzDn, UxDss, UyDss, UzDss, UxDds, UyDds, UzDds]
    hasS = !isempty(ExxDn); hasU = !isempty(UxDn)
    ref = hasS ? ExxDn : UxDn
    (hasS || hasU) || return (Sin[1:6]..., Uin[1:3]...)
    M, N = size(ref, 1), size(ref, 2)
    Sc = hasS ? [f64(a) for a in Sin] : Sin; Uc = hasU ? [f64(a) for a in Uin] : Uin
    So = [zeros(M, 1) for _ in 1:6]; Uo = [zeros(M, 1) for _ in 1:3]
    sip = [pointer(a) for a in Sc]; uip = [pointer(a) for a in Uc]
    sop = [pointer(a) for a in So]; uop = [pointer(a) for a in Uo]
    GC.@preserve Sc Uc So Uo sip uip sop uop begin
        check(ccall((:cad_td_sum, libcad), Cint,
            (Ptr{Cvoid}, Int64, Int64, Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}}),
            ctx(), M, N, hasS ? sip : C_NULL, hasU ? uip : C_NULL, hasS ? sop : C_NULL, hasU ? uop : C_NULL))
    end
    return ((hasS ? So : Sin[1:6])..., (hasU ? Uo : Uin[1:3])...)
end

# CalculateInfluenceMatrices3D (src/CalculateInfluenceMatrices3D.jl:2) -> TractionInf
function CalculateInfluenceMatrices3D(FaceNormalVector, MidPoint, P1, P2, P3, ν, G, λ, FixedEls, HSFlag, n)
    nf = count(!=(1), FixedEls)     # fixed elements: their columns are dropped
    T = [zeros(n, nf) for _ in 1:9]; tp = [pointer(a) for a in T]
    GC.@preserve T tp begin
        check(ccall((:cad_influence_traction, libcad), Cint,
            (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64,
             Float64, Float64, Float64, Ptr{Float64}, Cint, Ptr{Ptr{Float64}}),
            ctx(), f64(FaceNormalVector), f64(MidPoint), f64(P1), f64(P2), f64(P3), n, ν, G, λ,
            f64(vec(FixedEls)), HSFlag, tp))
    end
    return Ref_.TractionInf(T...)
end

# SlipCalculator3D (src/SlipCalculator3D.jl:1): the boundary conditions
# (Stresses, Tractions, MixedBoundaryConditions, ...) become (Tn, Tds, Tss)
# through the parent module's SetupTractionVector, as in the reference;
# returns Dn, Dss, Dds, A, b
function SlipCalculator3D(P1, P2, P3, ν, G, λ, MidPoint, FaceNormalVector, HSFlag, BoundaryConditions, FixedEls)
    n = length(FaceNormalVector[:, 1])
    (Tn, Tds, Tss) = Ref_.SetupTractionVector(BoundaryConditions, FaceNormalVector, n, G, λ)
    return any(FixedEls .== 1) ?
        slip_fixed(P1, P2, P3, ν, G, λ, MidPoint, FaceNormalVector, HSFlag, Tn, Tss, Tds, FixedEls) :
        slip_plain(P1, P2, P3, ν, G, λ, MidPoint, FaceNormalVector, HSFlag, Tn, Tss, Tds)
end

# plain system given (Tn, Tss, Tds): Dn, Dss, Dds, A, b
function slip_plain(P1, P2, P3, ν, G, λ, MidPoint, FaceNormalVector, HSFlag, Tn, Tss, Tds)
    n = size(P1, 1)
    Dn = zeros(n); Dss = zeros(n); Dds = zeros(n); A = zeros(3n, 3n); b = zeros(3n)
    check(ccall((:cad_slip_calculator, libcad), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Float64, Float64, Float64, Ptr{Float64},
         Ptr{Float64}, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
         Ptr{Float64}, Ptr{Float64}),
        ctx(), f64(P1), f64(P2), f64(P3), n, ν, G, λ, f64(MidPoint), f64(FaceNormalVector), HSFlag,
        f64(vec(Tn)), f64(vec(Tss)), f64(vec(Tds)), Dn, Dss, Dds, A, b))
    return Dn, Dss, Dds, A, b
end

# SlipCalculator3D with fixed elements (FixedEls .== 1): Dn, Dss, Dds of the
# other elements, A (3n x 3n_free), b
function slip_fixed(P1, P2, P3, ν, G, λ, MidPoint, FaceNormalVector, HSFlag, Tn, Tss, Tds, FixedEls)
    n = size(P1, 1)
    nf = count(!=(1), FixedEls)
    Dn = zeros(nf); Dss = zeros(nf); Dds = zeros(nf); A = zeros(3n, 3nf); b = zeros(3n)
    check(ccall((:cad_slip_calculator_fixed, libcad), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Float64, Float64, Float64, Ptr{Float64},
         Ptr{Float64}, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
         Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
        ctx(), f64(P1), f64(P2), f64(P3), n, ν, G, λ, f64(MidPoint), f64(FaceNormalVector), HSFlag,
        f64(vec(Tn)), f64(vec(Tss)), f64(vec(Tds)), f64(vec(FixedEls)), Dn, Dss, Dds, A, b))
    return Dn, Dss, Dds, A, b
end

# Frictional slip (src/SlipCalculator3D.jl:36-87): Tn, Tss, Tds are the element
# tractions of the MixedBoundaryConditions (remote stress resolved plus applied
# tractions), μ and Sf the FrictionParameters (one value or one per element).
# The reference's early exit (no element can overcome its frictional strength)
# is taken here as there.  The LCP is solved on the GPU (Fischer-Burmeister
# Newton in place of FischerNewton.fischer_newton, :196).
function SlipCalculator3D_friction(P1, P2, P3, ν, G, λ, MidPoint, FaceNormalVector, HSFlag, Tn, Tss, Tds, μ, Sf;
                                   tol::Real=1e-10, max_iter::Integer=100)
    n = size(P1, 1)
    μv = zeros(n) .+ μ
    Sfv = zeros(n) .+ Sf
    FricRes = vec(Tn) .* μv
    if all(-abs.(vec(Tss)) .> FricRes) && all(-abs.(vec(Tds)) .> FricRes)
        println("Cant overcome frictional strength")
        return zeros(n), zeros(n), zeros(n)
    end
    Dn = zeros(n); Dss = zeros(n); Dds = zeros(n)
    check(ccall((:cad_slip_calculator_friction, libcad), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Float64, Float64, Float64, Ptr{Float64},
         Ptr{Float64}, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Float64, Cint,
         Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
        ctx(), f64(P1), f64(P2), f64(P3), n, ν, G, λ, f64(MidPoint), f64(FaceNormalVector), HSFlag,
        f64(vec(Tn)), f64(vec(Tss)), f64(vec(Tds)), μv, Sfv, tol, max_iter, Dn, Dss, Dds))
    return Dn, Dss, Dds
end

# Prepared frictional system (src/SlipCalculator3D.jl:90-175 once, :177-238 per
# load): friction_prepare keeps C = inv(A Scl) on the GPU, friction_solve runs
# one load on it (no early exit, as in the reference's prepared overloads).
friction_prepare(P1, P2, P3, ν, G, λ, MidPoint, FaceNormalVector, HSFlag) =
    check(ccall((:cad_friction_prepare, libcad), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Float64, Float64, Float64, Ptr{Float64},
         Ptr{Float64}, Cint),
        ctx(), f64(P1), f64(P2), f64(P3), size(P1, 1), ν, G, λ, f64(MidPoint), f64(FaceNormalVector), HSFlag))

function friction_solve(Tn, Tss, Tds, μ, Sf; tol::Real=1e-10, max_iter::Integer=100)
    n = length(Tn)
    Dn = zeros(n); Dss = zeros(n); Dds = zeros(n)
    check(ccall((:cad_friction_solve, libcad), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Float64, Cint,
         Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
        ctx(), n, f64(vec(Tn)), f64(vec(Tss)), f64(vec(Tds)), zeros(n) .+ μ, zeros(n) .+ Sf, tol, max_iter,
        Dn, Dss, Dds))
    return Dn, Dss, Dds
end

# The LCP x ≥ 0, A x + b ≥ 0, x'(A x + b) = 0 (FischerNewton.fischer_newton(A, b)).
function fischer_newton(A, b; tol::Real=1e-10, max_iter::Integer=100)
    n = length(b)
    size(A) == (n, n) || error("DimensionMismatch: A must be $n x $n")
    x = zeros(n)
    check(ccall((:cad_fischer_newton, libcad), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Cint, Ptr{Float64}),
        ctx(), n, f64(A), f64(vec(b)), tol, max_iter, x))
    return x
end

# Precision settings (no counterpart in the reference): solver 0 = FP64 LU
# (default), 1 = FP32/TF32 LU + FP64 GMRES, 2 = FP64 GMRES with an installed
# block-sparse preconditioner, 3 = the same with the learned preconditioner
# built for each SlipCalculator3D mesh (network from set_network), 4 = FP64
# GMRES with element-block Jacobi, 5 = plain FP64 GMRES; assembly 0 = FP64,
# 1 = FP32 far field.
set_solver(mode::Integer, tol::Real=1e-10, max_iter::Integer=200) =
    check(ccall((:cad_set_solver, libcad), Cint, (Ptr{Cvoid}, Cint, Float64, Cint), ctx(), mode, tol, max_iter))
set_assembly(mode::Integer, near_factor::Real=3.0) =
    check(ccall((:cad_set_assembly, libcad), Cint, (Ptr{Cvoid}, Cint, Float64), ctx(), mode, near_factor))

# Learned preconditioner (no counterpart in the reference): the network's
# weights (Float32, cad_lpc_param_count of them), a training set built from
# meshes on the GPU, training, and installation for one mesh.
lpc_param_count() = ccall((:cad_lpc_param_count, libcad), Int64, ())
set_network(params::Vector{Float32}) =
    check(ccall((:cad_lpc_set_network, libcad), Cint, (Ptr{Cvoid}, Ptr{Float32}), ctx(), params))
function get_network()
    p = zeros(Float32, lpc_param_count())
    check(ccall((:cad_lpc_get_network, libcad), Cint, (Ptr{Cvoid}, Ptr{Float32}), ctx(), p))
    return p
end
dataset_add(P1, P2, P3, ν, G, λ, MidPoint, FaceNormalVector, HSFlag) =
    check(ccall((:cad_lpc_dataset_add, libcad), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Float64, Float64, Float64, Ptr{Float64},
         Ptr{Float64}, Cint),
        ctx(), f64(P1), f64(P2), f64(P3), size(P1, 1), ν, G, λ, f64(MidPoint), f64(FaceNormalVector), HSFlag))
function train(steps::Integer; batch::Integer=4096, lr::Real=1e-3, seed::Integer=0)
    hist = zeros(Float32, cld(steps, 100))
    check(ccall((:cad_lpc_train, libcad), Cint, (Ptr{Cvoid}, Int64, Int64, Float32, UInt64, Ptr{Float32}),
        ctx(), steps, batch, lr, seed, hist))
    return hist
end

# SlipCalculator3D over many independent cracks in one call: cracks is a vector
# of (P1, P2, P3, MidPoint, FaceNormalVector, Tn, Tss, Tds) tuples; returns a
# vector of (Dn, Dss, Dds) and the final relative residuals.
function SlipCalculator3D_batched(cracks, ν, G, λ, HSFlag)
    offs = Int64[0]
    for c in cracks
        push!(offs, offs[end] + size(c[1], 1))
    end
    cat(k) = reduce(vcat, [vec(f64(c[k])) for c in cracks])
    T = reduce(vcat, [vcat(vec(c[6]), vec(c[7]), vec(c[8])) for c in cracks])
    D = zeros(3 * offs[end]); rel = zeros(length(cracks))
    check(ccall((:cad_slip_calculator_batched, libcad), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
         Float64, Float64, Float64, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
        ctx(), length(cracks), offs, cat(1), cat(2), cat(3), cat(5), cat(4), ν, G, λ, HSFlag, T, D, rel))
    out = Vector{NTuple{3,Vector{Float64}}}()
    for c in 1:length(cracks)
        o = offs[c]; n = offs[c + 1] - o
        d = D[3o+1:3o+3n]
        push!(out, (d[1:n], d[n+1:2n], d[2n+1:3n]))
    end
    return out, rel
end

end # module
