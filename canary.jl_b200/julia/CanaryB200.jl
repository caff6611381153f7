# CanaryB200.jl — Julia binding of libcanary_b200.so (include/canary_b200.h).
#
# New methods of the reference's GPU-method names, dispatching on a device
# array type, so that the reference drivers (e.g. examples/3d_kernels/
# euler3d_set3c.jl:1227-1248, :1361-1523) run the sm_100a kernels unchanged.
# Arrays keep the reference layouts; pointers are device pointers.
module CanaryB200

using CUDA  # CuArray, CuPtr, CUDA.stream()
using MPI   # lowstorageRK_mpi

const libcb = joinpath(@__DIR__, "..", "lib", "libcanary_b200.so")

struct CbPhys
    gamma::Float64; R_gas::Float64; c_p::Float64; c_v::Float64
    gravity::Float64; Pr::Float64; lambda::Float64; visc::Float64
end
# reference constants (euler3d_set3c.jl:113-118, nse2d.jl:127-128)
const REFERENCE_PHYS = CbPhys(7/5, 287.17, 1004.67, 717.5, 10.0, 71/10, -2/3, 0.0)

function check(rc)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:cb_last_error, libcb), Cstring, ()))
    error("canary_b200 error $rc: $msg")
end

stream() = CUDA.stream().handle

function volumerhs!(::Val{dim}, ::Val{N}, rhs::CuArray{Float64}, Q, vgeo, D, elems;
                    phys = REFERENCE_PHYS) where {dim, N}
    check(ccall((:cb_volumerhs, libcb), Cint,
                (Cint, Cint, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64},
                 Int64, Ref{CbPhys}, Ptr{Cvoid}),
                dim, N, rhs, Q, vgeo, D, length(elems), phys, stream()))
end

function fluxrhs!(::Val{dim}, ::Val{N}, rhs::CuArray{Float64}, Q, sgeo, vgeo, elems, vmapM,
                  vmapP, elemtobndy; phys = REFERENCE_PHYS) where {dim, N}
    check(ccall((:cb_fluxrhs, libcb), Cint,
                (Cint, Cint, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64},
                 Int64, CuPtr{Int64}, CuPtr{Int64}, CuPtr{Int64}, Ref{CbPhys}, Ptr{Cvoid}),
                dim, N, rhs, Q, sgeo, vgeo, length(elems), vmapM, vmapP, elemtobndy, phys,
                stream()))
end

function updatesolution!(::Val{dim}, ::Val{N}, rhs::CuArray{Float64}, rhs_gradQ, Q, vgeo,
                         elems, rka, rkb, dt, visc) where {dim, N}
    check(ccall((:cb_updatesolution, libcb), Cint,
                (Cint, Cint, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64},
                 Int64, Float64, Float64, Float64, Float64, Ptr{Cvoid}),
                dim, N, rhs, visc > 0 ? rhs_gradQ : CU_NULL, Q, vgeo, length(elems), rka, rkb,
                dt, visc, stream()))
end

# lowstorageRK drop-in: fused stages, CUDA graph, state advanced in place.
function lowstorageRK(::Val{dim}, ::Val{N}, d_QL::CuArray{Float64}, d_rhsL, d_vgeoL, d_sgeo,
                      d_vmapM, d_vmapP, d_elemtobndy, d_D, dt, nsteps;
                      phys = REFERENCE_PHYS) where {dim, N}
    nelem = size(d_QL, 3)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:cb_solver_create, libcb), Cint,
                (Ref{Ptr{Cvoid}}, Cint, Cint, Cint, Int64, CuPtr{Float64}, CuPtr{Float64},
                 CuPtr{Float64}, CuPtr{Float64}, CuPtr{Int64}, CuPtr{Int64}, CuPtr{Int64},
                 CuPtr{Float64}, Ref{CbPhys}, Ptr{Cvoid}),
                h, dim, N, 64, nelem, d_QL, d_rhsL, d_vgeoL, d_sgeo, d_vmapM, d_vmapP,
                d_elemtobndy, d_D, phys, stream()))
    try
        check(ccall((:cb_lsrk_run, libcb), Cint, (Ptr{Cvoid}, Int64, Float64), h[], nsteps, dt))
    finally
        ccall((:cb_solver_destroy, libcb), Cint, (Ptr{Cvoid},), h[])
    end
    nothing
end

# Element-partitioned lowstorageRK over MPI ranks, with the reference's
# partition and ghost bookkeeping (connectmesh, src/mesh.jl:751-956:
# realelems then ghostelems, sendelems, nabrtorank / nabrtorecv /
# nabrtosend) and its exchange of whole elements before every stage
# (euler2d_set2c.jl:529-594, :707-735), through the ghosted solver's stage API.
# d_QL holds the real elements followed by the ghost elements; the MPI
# library must accept device buffers.
function lowstorageRK_mpi(::Val{dim}, ::Val{N}, mpicomm, d_QL::CuArray{Float64}, d_rhsL, d_vgeoL,
                          d_sgeo, d_vmapM, d_vmapP, d_elemtobndy, d_D, nrealelem, sendelems,
                          nabrtorank, nabrtorecv, nabrtosend, dt, nsteps;
                          phys = REFERENCE_PHYS) where {dim, N}
    nghost = size(d_QL, ndims(d_QL)) - nrealelem
    ew = length(d_QL) ÷ size(d_QL, ndims(d_QL))  # values per element
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:cb_solver_create_ghosted, libcb), Cint,
                (Ref{Ptr{Cvoid}}, Cint, Cint, Cint, Int64, Int64, CuPtr{Float64}, CuPtr{Float64},
                 CuPtr{Float64}, CuPtr{Float64}, CuPtr{Int64}, CuPtr{Int64}, CuPtr{Int64},
                 CuPtr{Float64}, Ref{CbPhys}, Ptr{Cvoid}),
                h, dim, N, 64, nrealelem, nghost, d_QL, d_rhsL, d_vgeoL, d_sgeo, d_vmapM, d_vmapP,
                d_elemtobndy, d_D, phys, stream()))
    sendidx = [CuArray{Int64}(sendelems[r] .- 1) for r in nabrtosend]  # 0-based own elements
    sendbuf = [CuArray{Float64}(undef, ew * length(r)) for r in nabrtosend]
    recvbuf = [CuArray{Float64}(undef, ew * length(r)) for r in nabrtorecv]
    next = Ref{Ptr{Cvoid}}(C_NULL)
    try
        for step in 1:nsteps, s in 0:4
            for n in eachindex(nabrtorank)
                check(ccall((:cb_solver_pack, libcb), Cint,
                            (Ptr{Cvoid}, Cint, CuPtr{Int64}, Int64, CuPtr{Float64}),
                            h[], 0, sendidx[n], length(sendidx[n]), sendbuf[n]))
            end
            CUDA.synchronize()
            reqs = MPI.Request[]
            for n in eachindex(nabrtorank)
                push!(reqs, MPI.Irecv!(recvbuf[n], nabrtorank[n], 777, mpicomm))
                push!(reqs, MPI.Isend(sendbuf[n], nabrtorank[n], 777, mpicomm))
            end
            MPI.Waitall!(reqs)
            for n in eachindex(nabrtorank)
                check(ccall((:cb_solver_unpack, libcb), Cint,
                            (Ptr{Cvoid}, Cint, CuPtr{Float64}, Int64, Int64),
                            h[], 0, recvbuf[n], first(nabrtorecv[n]) - nrealelem - 1,
                            length(nabrtorecv[n])))
            end
            check(ccall((:cb_solver_stage, libcb), Cint, (Ptr{Cvoid}, Cint, Float64, Ref{Ptr{Cvoid}}),
                        h[], s, dt, next))
        end
        check(ccall((:cb_solver_settle, libcb), Cint, (Ptr{Cvoid},), h[]))
    finally
        ccall((:cb_solver_destroy, libcb), Cint, (Ptr{Cvoid},), h[])
    end
    nothing
end

end # module
