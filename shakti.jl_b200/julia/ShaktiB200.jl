# ShaktiB200.jl -- the reference-side binding of libshakti_b200.so for Shakti.jl.
#
# UNTESTED: Julia is not available where this library was built and measured.  The C ABI it binds
# (include/shakti_b200.h) is exercised from Python (ctypes) by the test suite.
#
# Usage from a Shakti.jl session running with the CUDA backend:
#
#     using Shakti, CUDA
#     include("ShaktiB200.jl"); using .ShaktiB200
#     ls = B200CGSolver(grid; chebyshev_degree = 4)           # replaces CGIterativeSolver(grid, MatrixFreeLinearSystem; ...)
#     ps = PicardSolver(500, 1e-6, ls, grid)
#     sim = Simulation(grid, state, tsteps, dt, p, "implicit", String[], mi, sl; ps = ps)
#     run!(sim)                                              # Picard_iteration! dispatches to the method below
#
# The State's CuArrays are passed by pointer, with no copy: their layout is the library's layout.
module ShaktiB200

using CUDA
import Shakti
import Shakti: State, Grid, ModelParameters, AbstractIterativeSolver, AbstractKFaceScheme, Arithmetic, Harmonic,
               RegularizedCoulombSlidingLaw, RegularizedCoulombFieldSlidingLaw, RegularizedCoulombV0SlidingLaw,
               LinearSlidingLaw, PrescribedSlidingLaw, AbstractSlidingLaw

export B200CGSolver

const LIB = joinpath(@__DIR__, "..", "libshakti_b200.so")

# --- mirrors of the C structs (include/shakti_b200.h) -------------------------------------------
struct ShkParams
    rho_w::Float64; rho_sw::Float64; rho_i::Float64; g::Float64; nu::Float64; n::Float64; omega::Float64
    L::Float64; br::Float64; lr::Float64; ct::Float64; cw::Float64; p_atm::Float64; b_min::Float64
    b_max::Float64; e_v::Float64
end
ShkParams(p::ModelParameters) = ShkParams(p.rho_w, p.rho_sw, p.rho_i, p.g, p.nu, p.n, p.omega, p.L, p.br, p.lr,
                                          p.ct, p.cw, p.p_atm, p.b_min, p.b_max, p.e_v)

struct ShkSliding
    kind::Cint; C::Float64; v0::Float64; Cx::Ptr{Float64}; Cy::Ptr{Float64}
end
ShkSliding(sl::RegularizedCoulombSlidingLaw) = ShkSliding(0, sl.C, 0.0, C_NULL, C_NULL)
ShkSliding(sl::RegularizedCoulombFieldSlidingLaw) = ShkSliding(1, 0.0, 0.0, pointer(sl.Cx), pointer(sl.Cy))
ShkSliding(sl::RegularizedCoulombV0SlidingLaw) = ShkSliding(2, 0.0, sl.v0, pointer(sl.Cx), pointer(sl.Cy))
ShkSliding(sl::LinearSlidingLaw) = ShkSliding(3, 0.0, 0.0, pointer(sl.Cx2), pointer(sl.Cy2))
ShkSliding(::PrescribedSlidingLaw) = ShkSliding(4, 0.0, 0.0, C_NULL, C_NULL)

struct ShkCgOpts
    precond::Cint; cheb_degree::Cint; cheb_nsteps::Cint; stop_rule::Cint; precision::Cint; max_refine::Cint
    atol::Float64; rtol::Float64; inner_rtol::Float64; itmax::Clong; inner_itmax::Clong
end

mutable struct ShkCgStats
    niter::Clong; status::Cint; refinements::Cint; rnorm0::Float64; rnorm::Float64
    lambda_min::Float64; lambda_max::Float64; bounds_valid::Cint
    ShkCgStats() = new(0, 0, 0, 0.0, 0.0, 1.0, 1.0, 0)
end

# State field order of shk_state (src/state.jl:13-57)
const STATE_FIELDS = (:h, :pw, :po, :b, :beta, :abs_ub, :mdot, :shear, :potential, :sensible, :Re, :K, :G, :zb,
                      :zs, :H, :ieb, :lambda, :A_visc, :N, :mask,
                      :dhdx, :q_x, :Re_x, :b_x, :ub_x, :taub_x, :dpwdx, :valid_x,
                      :dhdy, :q_y, :Re_y, :b_y, :ub_y, :taub_y, :dpwdy, :valid_y)
state_pointers(s::State) = [reinterpret(Ptr{Float64}, pointer(getfield(s, f))) for f in STATE_FIELDS]

check(ctx, rc, ok = (0,)) = rc in ok ? rc :
    error("libshakti_b200: ", unsafe_string(ccall((:shk_last_error, LIB), Cstring, (Ptr{Cvoid},), ctx)))

# --- the solver object: replaces CGIterativeSolver(g, MatrixFreeLinearSystem; ...) ---------------
mutable struct B200CGSolver <: AbstractIterativeSolver
    ctx::Ptr{Cvoid}
    opts::ShkCgOpts
    stats::ShkCgStats
end

function B200CGSolver(g::Grid; chebyshev_degree::Union{Nothing, Int} = nothing, chebyshev_nsteps_estimate::Int = 15,
                      atol = sqrt(eps(Float64)), rtol = sqrt(eps(Float64)), itmax::Int = 0)
    ctxref = Ref{Ptr{Cvoid}}(C_NULL)
    stream = CUDA.stream().handle
    rc = ccall((:shk_create, LIB), Cint, (Cint, Cint, Float64, Float64, Ptr{Cvoid}, Ref{Ptr{Cvoid}}),
               g.nx, g.ny, g.lx, g.ly, stream, ctxref)
    rc == 0 || error("shk_create failed with status $rc")
    cheb = chebyshev_degree !== nothing
    opts = ShkCgOpts(cheb ? 1 : 0, cheb ? chebyshev_degree : 4, chebyshev_nsteps_estimate, 0, 0, 0, atol, rtol,
                     0.0, itmax, 0)
    ls = B200CGSolver(ctxref[], opts, ShkCgStats())
    finalizer(x -> ccall((:shk_destroy, LIB), Cint, (Ptr{Cvoid},), x.ctx), ls)
    return ls
end

function bind!(ls::B200CGSolver, s::State, p::ModelParameters, sl::AbstractSlidingLaw, kfs::AbstractKFaceScheme)
    ctx = ls.ctx
    check(ctx, ccall((:shk_set_stream, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), ctx, CUDA.stream().handle))
    check(ctx, ccall((:shk_set_params, LIB), Cint, (Ptr{Cvoid}, Ref{ShkParams}), ctx, ShkParams(p)))
    check(ctx, ccall((:shk_set_sliding_law, LIB), Cint, (Ptr{Cvoid}, Ref{ShkSliding}), ctx, ShkSliding(sl)))
    check(ctx, ccall((:shk_set_schemes, LIB), Cint, (Ptr{Cvoid}, Cint, Cint), ctx, kfs isa Harmonic ? 1 : 0, 1))
    ptrs = state_pointers(s)
    check(ctx, ccall((:shk_bind_state, LIB), Cint, (Ptr{Cvoid}, Ptr{Ptr{Float64}}), ctx, ptrs))
    return ls
end

# solve_elliptic_linear_system!(ls, s, g, p, kfs) (src/linear_solver.jl:915-925)
function Shakti.solve_elliptic_linear_system!(ls::B200CGSolver, s::State, g::Grid, p::ModelParameters,
                                              kfs::AbstractKFaceScheme)
    bind!(ls, s, p, RegularizedCoulombSlidingLaw(0.0), kfs)
    rc = ccall((:shk_solve_elliptic, LIB), Cint, (Ptr{Cvoid}, Ref{ShkCgOpts}, Ref{ShkCgStats}), ls.ctx, ls.opts,
               ls.stats)
    check(ls.ctx, rc, (0, 1, 2))
    return s
end

# solve_parabolic_linear_system!(ls, s, g, p, kfs, dt) (src/linear_solver.jl:935-945)
function Shakti.solve_parabolic_linear_system!(ls::B200CGSolver, s::State, g::Grid, p::ModelParameters,
                                               kfs::AbstractKFaceScheme, dt)
    bind!(ls, s, p, RegularizedCoulombSlidingLaw(0.0), kfs)
    rc = ccall((:shk_solve_parabolic, LIB), Cint, (Ptr{Cvoid}, Float64, Ref{ShkCgOpts}, Ref{ShkCgStats}), ls.ctx,
               Float64(dt), ls.opts, ls.stats)
    check(ls.ctx, rc, (0, 1, 2))
    return s
end

end # module
