/*
 * mpi-ext.h stand-in (oracle test infrastructure only): the Fujitsu MPI
 * topology extension that the reference's ring/bucket code calls
 * (lib/libbine_common.cc:2499-2506, lib/libbine_coll_allgather.cc:1349-1432).
 * That code is Fugaku-only and never selected by the oracle; every call here
 * reports failure.
 */
#ifndef BINE_MPISHIM_MPI_EXT_H
#define BINE_MPISHIM_MPI_EXT_H

#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FJMPI_SUCCESS 0
#define FJMPI_ERR_TOPOLOGY 1
#define FJMPI_LOGICAL 0
#define FJMPI_PHYSICAL 1

int FJMPI_Topology_get_dimension(int *size);
int FJMPI_Topology_get_shape(int *x, int *y, int *z);
int FJMPI_Topology_get_coords(MPI_Comm comm, int rank, int view, int maxdims, int coords[]);
int FJMPI_Topology_get_ranks(MPI_Comm comm, int view, int coords[], int maxppn, int *outppn, int ranks[]);

#ifdef __cplusplus
}
#endif

#endif /* BINE_MPISHIM_MPI_EXT_H */
