/*
 * Single-process stand-in for the subset of MPI that SHOCK's hot-path
 * translation units reference (Functions.c, WENO.c, ZD.c, BC.c,
 * ManufacturedSolution.c).  Only the declarations live here; the
 * definitions are in mpi_stub.c.  Test infrastructure for the reference
 * build under oracle/_ref -- not part of the shipped library.
 */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H

typedef int MPI_Comm;
typedef int MPI_Info;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_File;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_FLOAT 1
#define MPI_DOUBLE 2
#define MPI_LONG_DOUBLE 3
#define MPI_INT 4
#define MPI_CHAR 5
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_TAG_UB 1
#define MPI_PROC_NULL (-2)
#define MPI_REQUEST_NULL 0
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_ORDER_C 0
#define MPI_MODE_RDONLY 2
#define MPI_MAJOR_VERSION 3
#define MPI_MINOR_VERSION 0
#define MPI_RELEASE_VERSION 0

int MPI_Init(int *, char ***);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm, int *);
int MPI_Comm_rank(MPI_Comm, int *);
int MPI_Barrier(MPI_Comm);
double MPI_Wtime(void);
int MPI_Abort(MPI_Comm, int);
int MPI_Comm_get_attr(MPI_Comm, int, void *, int *);
int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *);
int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *);
int MPI_Test(MPI_Request *, int *, MPI_Status *);
int MPI_Waitall(int, MPI_Request *, MPI_Status *);
int MPI_Sendrecv(const void *, int, MPI_Datatype, int, int, void *, int,
                 MPI_Datatype, int, int, MPI_Comm, MPI_Status *);
int MPI_Allgather(const void *, int, MPI_Datatype, void *, int, MPI_Datatype, MPI_Comm);
int MPI_Reduce(const void *, void *, int, MPI_Datatype, MPI_Op, int, MPI_Comm);
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm);
int MPI_Cart_create(MPI_Comm, int, const int *, const int *, int, MPI_Comm *);
int MPI_Cart_coords(MPI_Comm, int, int, int *);
int MPI_Cart_shift(MPI_Comm, int, int, int *, int *);
int MPI_Type_create_subarray(int, const int *, const int *, const int *, int,
                             MPI_Datatype, MPI_Datatype *);
int MPI_Type_commit(MPI_Datatype *);
int MPI_Type_size(MPI_Datatype, int *);
/* MPI-IO, read-only: what loadDivision (src/Load.c:191-250) calls; defined
   in mpi_shm.c only. */
int MPI_File_open(MPI_Comm, const char *, int, MPI_Info, MPI_File *);
int MPI_File_get_size(MPI_File, MPI_Offset *);
int MPI_File_set_view(MPI_File, MPI_Offset, MPI_Datatype, MPI_Datatype, const char *, MPI_Info);
int MPI_File_read(MPI_File, void *, int, MPI_Datatype, MPI_Status *);
int MPI_File_close(MPI_File *);

#endif
