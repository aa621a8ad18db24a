# StokesFlowB200.jl -- drop-in replacements for the hot-path functions of
# StokesFlow.jl (dastrm/StokesFlow.jl), calling libstokesflow_b200.so through
# `ccall`.  Each method keeps the reference's name, signature, argument
# meaning and in-place behaviour; the arrays must be CUDA.jl `CuArray{Float64}`
# (column-major, as the reference's `Data.Array` on the GPU backend).
#
#   include("StokesFlowB200.jl"); using .StokesFlowB200
#
# then call bilinearMarkerToGrid!, solveStokes! and moveMarkersRK4! exactly as
# scripts/StokesFlow2D_multixpu.jl:164-181 does.  exchangeMarkers is the
# identity on a single domain and needs no replacement.
#
# This file is written against the C ABI in include/stokesflow_b200.h.  There
# is no Julia toolchain on the build machine, so it has not been executed;
# the same ABI is exercised by the Python binding and the tests.
module StokesFlowB200

using CUDA

export bilinearMarkerToGrid!, bilinearMarkerToGrids!, solveStokes!, moveMarkersRK4!, solveStokesMixed!

const libsf = joinpath(@__DIR__, "..", "lib", "libstokesflow_b200.so")

struct SolveInfo
    dt::Float64
    T_eff::Float64
    runtime::Float64
    iters::Int64
    err::Float64
    n_checks::Int64
    converged::Int32
    reserved::Int32
    loop_ms::Float64
    bytes_per_iter::Float64
    T_eff_essential::Float64
    fused_launches::Int64
    fused_ms::Float64
end

const _ctx = Ref{Ptr{Cvoid}}(C_NULL)

function ctx()
    if _ctx[] == C_NULL
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:sf_ctx_create, libsf), Cint, (Cint, Ref{Ptr{Cvoid}}), CUDA.deviceid(CUDA.device()), h))
        _ctx[] = h[]
    end
    return _ctx[]
end

function check(status::Cint)
    status == 0 && return nothing
    msg = unsafe_string(ccall((:sf_last_error, libsf), Cstring, ()))
    status == 1 ? throw(AssertionError(msg)) : error("libstokesflow_b200: " * msg)
end

dptr(A::CuArray{Float64}) = reinterpret(Ptr{Cdouble}, pointer(A))
dptr(::Nothing) = Ptr{Cdouble}(C_NULL)
stream() = CUDA.stream().handle

# MarkerToGrid.jl:18
function bilinearMarkerToGrid!(x_grid_min, y_grid_min, val_grid, x_m, y_m, val_m, dx, dy, val_wt_sum, wt_sum, grid)
    Nx, Ny = size(val_grid)
    Nm = size(x_m, 1)
    @assert (size(y_m, 1) == Nm) && (size(val_m, 1) == Nm)
    check(ccall((:sf_bilinear_marker_to_grid, libsf), Cint,
                (Ptr{Cvoid}, Cdouble, Cdouble, Ptr{Cdouble}, Int64, Int64, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                 Int64, Cdouble, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Int64, Int64, Ptr{Cvoid}),
                ctx(), x_grid_min, y_grid_min, dptr(val_grid), Nx, Ny, dptr(x_m), dptr(y_m), dptr(val_m), Nm, dx, dy,
                dptr(val_wt_sum), dptr(wt_sum), size(wt_sum, 1), length(wt_sum), stream()))
    return nothing
end

# one grid of bilinearMarkerToGrids!: sf_deposit_grid
struct DepositGrid
    x_grid_min::Float64; y_grid_min::Float64
    val_grid::Ptr{Cdouble}
    nx::Int64; ny::Int64
    val_m::Ptr{Cdouble}
end

# The deposits of one timestep (StokesFlow2D_multixpu.jl:164-166) in one call: grids is a list of
# (x_grid_min, y_grid_min, val_grid, val_m); same result as bilinearMarkerToGrid! once per grid in order.
function bilinearMarkerToGrids!(grids, x_m, y_m, dx, dy, val_wt_sum, wt_sum)
    Nm = size(x_m, 1)
    @assert size(y_m, 1) == Nm && all(size(g[4], 1) == Nm for g in grids)
    GC.@preserve grids begin
        gs = [DepositGrid(g[1], g[2], dptr(g[3]), size(g[3], 1), size(g[3], 2), dptr(g[4])) for g in grids]
        check(ccall((:sf_bilinear_marker_to_grids, libsf), Cint,
                    (Ptr{Cvoid}, Ptr{DepositGrid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Int64, Cdouble, Cdouble,
                     Ptr{Cdouble}, Ptr{Cdouble}, Int64, Int64, Ptr{Cvoid}),
                    ctx(), gs, length(gs), dptr(x_m), dptr(y_m), Nm, dx, dy, dptr(val_wt_sum), dptr(wt_sum),
                    size(wt_sum, 1), length(wt_sum), stream()))
    end
    return nothing
end

# StokesSolver_multixpu.jl:14-15
function solveStokes!(P, Vx_pad, Vy_pad, ρ_vy, μ_b, μ_p, τxx, τyy, τxy, ∇V, dτPt, Rx, Ry, dVxdτ, dVydτ, dτVx, dτVy,
                      Vx_s, Vy_s, g_y, dx, dy, Nx, Ny, dt, maxdisp, comm; use_free_surface_stabilization::Bool=true,
                      ϵ=1e-8, print_info::Bool=true, iterMax=100000)
    info = Ref{SolveInfo}()
    check(ccall((:sf_solve_stokes, libsf), Cint,
                (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                 Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                 Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                 Cdouble, Cdouble, Cdouble, Int64, Int64, Cdouble, Cdouble, Cint, Cdouble, Cint, Int64, Ptr{Cvoid},
                 Ref{SolveInfo}),
                ctx(), dptr(P), dptr(Vx_pad), dptr(Vy_pad), dptr(ρ_vy), dptr(μ_b), dptr(μ_p), dptr(τxx), dptr(τyy),
                dptr(τxy), dptr(∇V), dptr(dτPt), dptr(Rx), dptr(Ry), dptr(dVxdτ), dptr(dVydτ), dptr(dτVx), dptr(dτVy),
                dptr(Vx_s), dptr(Vy_s), g_y, dx, dy, Nx, Ny, dt, maxdisp, use_free_surface_stabilization, ϵ,
                print_info, iterMax, stream(), info))
    return info[].dt, info[].T_eff, info[].runtime
end

# sf_batch_instance: one problem of the mixed-precision / batched solver, results written back
struct BatchInstance
    P::Ptr{Cdouble}; Vx_pad::Ptr{Cdouble}; Vy_pad::Ptr{Cdouble}; ρ_vy::Ptr{Cdouble}; μ_b::Ptr{Cdouble}
    μ_p::Ptr{Cdouble}; Vx_s::Ptr{Cdouble}; Vy_s::Ptr{Cdouble}
    Nx::Int64; Ny::Int64
    g_y::Float64; dx::Float64; dy::Float64; dt::Float64; maxdisp::Float64; eps::Float64; rel_tol::Float64
    use_free_surface_stabilization::Int32; retried::Int32
    dt_out::Float64; err::Float64; eps_used::Float64
    inner_iters::Int64; outer_iters::Int64
    converged::Int32; status::Int32
    batch_ms::Float64
    dVxdt::Ptr{Cdouble}; dVydt::Ptr{Cdouble}
end

# The problem of solveStokes! solved by FP32 pseudo-transient sweeps with FP64 defect correction: the same
# FP64 stopping test and iteration schedule, not the same bits.  dVxdτ, dVydτ are the damped rates, carried
# from call to call as solveStokes! carries them.  Returns (dt, err, FP32 sweeps).  rel_tol > 0 replaces ϵ by
# rel_tol * mean|g_y ρ_vy|.
function solveStokesMixed!(P, Vx_pad, Vy_pad, ρ_vy, μ_b, μ_p, Vx_s, Vy_s, dVxdτ, dVydτ, g_y, dx, dy, Nx, Ny, dt,
                           maxdisp; use_free_surface_stabilization::Bool=true, ϵ=1e-8, rel_tol=0.0)
    info = Ref{BatchInstance}()
    check(ccall((:sf_solve_stokes_mixed, libsf), Cint,
                (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                 Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Cdouble, Cdouble, Cdouble, Int64, Int64,
                 Cdouble, Cdouble, Cint, Cdouble, Cdouble, Ptr{Cvoid}, Ptr{Cvoid}, Ref{BatchInstance}),
                ctx(), dptr(P), dptr(Vx_pad), dptr(Vy_pad), dptr(ρ_vy), dptr(μ_b), dptr(μ_p), dptr(Vx_s), dptr(Vy_s),
                dptr(dVxdτ), dptr(dVydτ), g_y, dx, dy, Nx, Ny, dt, maxdisp, use_free_surface_stabilization, ϵ,
                rel_tol, C_NULL, stream(), info))
    return info[].dt_out, info[].err, info[].inner_iters
end

# MoveMarkers.jl:15
function moveMarkersRK4!(x_m, y_m, Vx, Vy, x_vx_min, y_vx_min, x_vy_min, y_vy_min, dt, lx, ly, dx, dy)
    Nm = length(x_m)
    @assert (Nm == length(y_m)) "x and y Marker coords have not same length"
    check(ccall((:sf_move_markers_rk4, libsf), Cint,
                (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Int64, Ptr{Cdouble}, Int64, Int64, Ptr{Cdouble}, Int64, Int64,
                 Cdouble, Cdouble, Cdouble, Cdouble, Cdouble, Cdouble, Cdouble, Cdouble, Cdouble, Ptr{Cvoid}),
                ctx(), dptr(x_m), dptr(y_m), Nm, dptr(Vx), size(Vx, 1), size(Vx, 2), dptr(Vy), size(Vy, 1),
                size(Vy, 2), x_vx_min, y_vx_min, x_vy_min, y_vy_min, dt, lx, ly, dx, dy, stream()))
    return nothing
end

end # module
