// Single-rank stand-in for <mpi.h>, used only to compile the reference
// solver's own sources into the CPU oracle harness and the CPU baseline.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product links against it.
//
// Every call behaves as MPI does on a communicator of size one: the process
// is rank 0, Cartesian neighbours are MPI_PROC_NULL, collectives copy the
// send buffer into the receive buffer.  MPI_Abort hands its error code to
// dsmc_ref_mpi_abort(), which the harness turns into a C++ exception (so a
// test process survives) and the baseline program turns into exit(code).
#pragma once

#include <cstddef>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef std::ptrdiff_t MPI_Aint;

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0
#define MPI_SUM 1

#define MPI_INT 1
#define MPI_DOUBLE 2

[[noreturn]] void dsmc_ref_mpi_abort(int code);

namespace dsmc_mpi_stub {
// Byte extent of each datatype handle; derived types get the next free slot.
inline std::size_t extents[64] = {0, sizeof(int), sizeof(double)};
inline int next_type = 3;

inline std::size_t bytes(MPI_Datatype t, long count)
{
    return extents[t] * static_cast<std::size_t>(count);
}

inline void copy(void *dst, const void *src, std::size_t n)
{
    if (n != 0 && dst != nullptr && src != nullptr && dst != src)
        std::memmove(dst, src, n);
}
} // namespace dsmc_mpi_stub

inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
inline int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int code) { dsmc_ref_mpi_abort(code); }

inline int MPI_Type_create_struct(int, const int *, const MPI_Aint *, const MPI_Datatype *,
                                  MPI_Datatype *out)
{
    *out = dsmc_mpi_stub::next_type++;
    dsmc_mpi_stub::extents[*out] = 0;
    return MPI_SUCCESS;
}

inline int MPI_Type_create_resized(MPI_Datatype, MPI_Aint, MPI_Aint extent, MPI_Datatype *out)
{
    *out = dsmc_mpi_stub::next_type++;
    dsmc_mpi_stub::extents[*out] = static_cast<std::size_t>(extent);
    return MPI_SUCCESS;
}

inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype *) { return MPI_SUCCESS; }

inline int MPI_Dims_create(int, int ndims, int *dims)
{
    for (int i = 0; i < ndims; ++i)
        if (dims[i] == 0)
            dims[i] = 1;
    return MPI_SUCCESS;
}

inline int MPI_Cart_create(MPI_Comm, int, const int *, const int *, int, MPI_Comm *out)
{
    *out = MPI_COMM_WORLD;
    return MPI_SUCCESS;
}

inline int MPI_Cart_coords(MPI_Comm, int, int maxdims, int *coords)
{
    for (int i = 0; i < maxdims; ++i)
        coords[i] = 0;
    return MPI_SUCCESS;
}

inline int MPI_Cart_shift(MPI_Comm, int, int, int *source, int *dest)
{
    *source = MPI_PROC_NULL;
    *dest = MPI_PROC_NULL;
    return MPI_SUCCESS;
}

inline int MPI_Cart_rank(MPI_Comm, const int *, int *rank) { *rank = 0; return MPI_SUCCESS; }

inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, int,
                      MPI_Comm)
{
    dsmc_mpi_stub::copy(recv, send, dsmc_mpi_stub::bytes(type, count));
    return MPI_SUCCESS;
}

inline int MPI_Alltoall(const void *send, int scount, MPI_Datatype stype, void *recv, int,
                        MPI_Datatype, MPI_Comm)
{
    dsmc_mpi_stub::copy(recv, send, dsmc_mpi_stub::bytes(stype, scount));
    return MPI_SUCCESS;
}

inline int MPI_Alltoallv(const void *send, const int *scounts, const int *sdispls,
                         MPI_Datatype stype, void *recv, const int *, const int *rdispls,
                         MPI_Datatype rtype, MPI_Comm)
{
    if (send == nullptr || recv == nullptr)
        return MPI_SUCCESS;
    const char *s = static_cast<const char *>(send) + dsmc_mpi_stub::bytes(stype, sdispls[0]);
    char *r = static_cast<char *>(recv) + dsmc_mpi_stub::bytes(rtype, rdispls[0]);
    dsmc_mpi_stub::copy(r, s, dsmc_mpi_stub::bytes(stype, scounts[0]));
    return MPI_SUCCESS;
}

inline int MPI_Gather(const void *send, int scount, MPI_Datatype stype, void *recv, int,
                      MPI_Datatype, int, MPI_Comm)
{
    dsmc_mpi_stub::copy(recv, send, dsmc_mpi_stub::bytes(stype, scount));
    return MPI_SUCCESS;
}

inline int MPI_Gatherv(const void *send, int scount, MPI_Datatype stype, void *recv,
                       const int *, const int *displs, MPI_Datatype rtype, int, MPI_Comm)
{
    if (recv == nullptr)
        return MPI_SUCCESS;
    char *r = static_cast<char *>(recv) + dsmc_mpi_stub::bytes(rtype, displs[0]);
    dsmc_mpi_stub::copy(r, send, dsmc_mpi_stub::bytes(stype, scount));
    return MPI_SUCCESS;
}
