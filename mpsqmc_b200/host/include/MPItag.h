// Multi-process switch of the reference (include/MPItag.h).  This build runs one process per
// GPU and never defines USE_MPI_IN_MPSQMC.
