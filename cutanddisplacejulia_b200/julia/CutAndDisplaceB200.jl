# CutAndDisplaceB200 — Julia bindings of libcad_td.so (the B200 TD path).
#
# Drop-in replacements for CutAndDisplaceJulia's TD, TD_sum,
# CalculateInfluenceMatrices3D and the plain SlipCalculator3D: same names,
# argument order and meaning, same struct field orders, same error texts.
# Each method checks dimensions as the reference does, then ccalls the C ABI
# declared in include/cad_td.h.  Usage inside CutAndDisplaceJulia:
#
#     include("CutAndDisplaceB200.jl"); using .CutAndDisplaceB200
#     # then call TD / TD_sum / CalculateInfluenceMatrices3D / SlipCalculator3D
#     # through this module in place of the reference's methods
module CutAndDisplaceB200

const libcad = get(ENV, "CAD_TD_LIB", joinpath(@__DIR__, "..", "libcad_td.so"))

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

# TD: influence-matrix overload (returns StrainInf, DispInf as NamedTuples of M x N matrices)
function TD(X, Y, Z, P1, P2, P3, Dss, Dds, Dn, ν, G, DispFlag, StrainFlag, HSflag)
    dims_ok(P1, P2, P3, Dss, Dds, Dn) || error("Element size inputs must be the same dimensions")
    M = length(X); N = length(P1) == 3 ? 1 : size(P1, 1)
    S = StrainFlag == 1 ? [zeros(M, N) for _ in 1:18] : [Float64[] for _ in 1:18]
    U = DispFlag == 1 ? [zeros(M, N) for _ in 1:9] : [Float64[] for _ in 1:9]
    sp = [pointer(a) for a in S]; up = [pointer(a) for a in U]
    GC.@preserve S U sp up begin
        check(ccall((:cad_td_inf, libcad), Cint,
            (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
             Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Cint, Cint, Cint,
             Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}}),
            ctx(), f64(vec(X)), f64(vec(Y)), f64(vec(Z)), M, f64(P1), f64(P2), f64(P3), N,
            f64(vec(Dss)), f64(vec(Dds)), f64(vec(Dn)), ν, G, DispFlag, StrainFlag, HSflag,
            StrainFlag == 1 ? sp : C_NULL, DispFlag == 1 ? up : C_NULL))
    end
    return S, U
end

# TD: summing overload -> (εxx, εyy, εzz, εxy, εxz, εyz), (Ux, Uy, Uz) reshaped like X
function TD_summed(X, Y, Z, P1, P2, P3, Dss, Dds, Dn, ν, G, DispFlag, StrainFlag, HSflag)
    dims_ok(P1, P2, P3, Dss, Dds, Dn) || error("Element size inputs must be the same dimensions")
    M = length(X); N = length(P1) == 3 ? 1 : size(P1, 1)
    S = [zeros(M) for _ in 1:6]; U = [zeros(M) for _ in 1:3]
    sp = [pointer(a) for a in S]; up = [pointer(a) for a in U]
    GC.@preserve S U sp up begin
        check(ccall((:cad_td_sum_eval, libcad), Cint,
            (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
             Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Cint, Cint, Cint,
             Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}}),
            ctx(), f64(vec(X)), f64(vec(Y)), f64(vec(Z)), M, f64(P1), f64(P2), f64(P3), N,
            f64(vec(Dss)), f64(vec(Dds)), f64(vec(Dn)), ν, G, DispFlag, StrainFlag, HSflag, sp, up))
    end
    shape = size(X, 2) != 1 ? size(X) : (M,)
    return [reshape(a, shape) for a in S], [reshape(a, shape) for a in U]
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

# CalculateInfluenceMatrices3D -> nine n x n matrices in TractionInf field order
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
    return T
end

# Plain SlipCalculator3D given (Tn, Tss, Tds): returns Dn, Dss, Dds, A, b
function SlipCalculator3D(P1, P2, P3, ν, G, λ, MidPoint, FaceNormalVector, HSFlag, Tn, Tss, Tds)
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
function SlipCalculator3D(P1, P2, P3, ν, G, λ, MidPoint, FaceNormalVector, HSFlag, Tn, Tss, Tds, FixedEls)
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
# (default), 1 = FP32/TF32 LU + FP64 GMRES, 2 = FP64 GMRES with the block-sparse
# preconditioner set below; assembly 0 = FP64, 1 = FP32 far field.
set_solver(mode::Integer, tol::Real=1e-10, max_iter::Integer=200) =
    check(ccall((:cad_set_solver, libcad), Cint, (Ptr{Cvoid}, Cint, Float64, Cint), ctx(), mode, tol, max_iter))
set_assembly(mode::Integer, near_factor::Real=3.0) =
    check(ccall((:cad_set_assembly, libcad), Cint, (Ptr{Cvoid}, Cint, Float64), ctx(), mode, near_factor))

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
