/* Single-rank stand-in for the subset of the MPI API that SPM-IQC's sources
 * call (MPI_Init/Finalize/Comm_size/Comm_rank/Barrier/Wtime/Bcast/Reduce/
 * Allreduce/Scatter/Gather). TEST INFRASTRUCTURE ONLY: it lets the reference's
 * own src/*.cpp compile unchanged as the CPU oracle. With one rank every
 * collective is a copy (or a no-op), which is exactly what MPICH does for a
 * communicator of size 1.
 *
 * Call sites served: src/LPsrc.cpp:55,87,93,165; src/BasicOperators.cpp:140,153;
 * src/LOBPCG.cpp:72,145,190,353,433; src/SPM.cpp:75,144,289; src/My_FFT.cpp:75,119.
 */
#ifndef SPMIQC_ORACLE_SHIM_MPI_H
#define SPMIQC_ORACLE_SHIM_MPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0

/* datatype codes: value = element size in bytes so the shim can copy */
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_C_DOUBLE_COMPLEX 16

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LOR 4

#define MPI_IN_PLACE ((void *)1)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
               MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm);
int MPI_Scatter(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                void *recvbuf, int recvcount, MPI_Datatype recvtype, int root,
                MPI_Comm comm);
int MPI_Gather(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
               void *recvbuf, int recvcount, MPI_Datatype recvtype, int root,
               MPI_Comm comm);

#ifdef __cplusplus
}
#endif

#endif
