/* Single-process stand-in for the MPI declarations the reference's CUDA files
 * name (src/Core/ControlCUDA.cpp:14, src/Core/DiagnosticCUDA.cpp:13).  The
 * oracle/_ref build runs one rank with MPISingle set, so none of these is
 * called; each is defined to fail loudly.  Test infrastructure. */
#ifndef G4REF_UPSTREAM_MPI_H_
#define G4REF_UPSTREAM_MPI_H_
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int source, tag, error; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_SUM 2
int MPI_Comm_size(MPI_Comm, int*);
int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm);
int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm);
int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*);
int MPI_Abort(MPI_Comm, int);
#endif
