/* Single-rank stand-in for <mpi.h>, used only to compile reference sources
 * for the oracle pins (oracle/ref_build.sh).  Collectives copy their input. */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H
#include <string.h>
typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Status;
typedef int MPI_Op;
#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_MAX_ERROR_STRING 64
#define MPI_DATATYPE_NULL 0
#define MPI_STATUS_IGNORE 0
#define MPI_STATUSES_IGNORE 0
#define MPI_MAX 1
enum { MPI_CHAR = 1, MPI_SIGNED_CHAR, MPI_UNSIGNED_CHAR, MPI_WCHAR, MPI_SHORT, MPI_UNSIGNED_SHORT,
       MPI_INT, MPI_UNSIGNED, MPI_LONG, MPI_UNSIGNED_LONG, MPI_LONG_LONG, MPI_UNSIGNED_LONG_LONG,
       MPI_FLOAT, MPI_DOUBLE, MPI_LONG_DOUBLE, MPI_INT8_T, MPI_INT16_T, MPI_INT32_T, MPI_INT64_T,
       MPI_UINT8_T, MPI_UINT16_T, MPI_UINT32_T, MPI_UINT64_T, MPI_C_BOOL, MPI_C_COMPLEX,
       MPI_C_FLOAT_COMPLEX, MPI_C_DOUBLE_COMPLEX, MPI_C_LONG_DOUBLE_COMPLEX };
static inline int shim_mpi_size(int t) { return t == MPI_DOUBLE ? 8 : t == MPI_FLOAT ? 4 : t == MPI_INT ? 4 : 8; }
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Barrier(int) { return 0; }
static inline int MPI_Comm_size(int, int *s) { *s = 1; return 0; }
static inline int MPI_Comm_rank(int, int *r) { *r = 0; return 0; }
static inline int MPI_Error_class(int, int *) { return 0; }
static inline int MPI_Error_string(int, char *, int *) { return 0; }
static inline int MPI_Abort(int, int) { return 0; }
static inline int MPI_Isend(const void *, int, int, int, int, int, int *) { return 0; }
static inline int MPI_Irecv(void *, int, int, int, int, int, int *) { return 0; }
static inline int MPI_Waitall(int, int *, int) { return 0; }
static inline int MPI_Allreduce(const void *in, void *out, int count, int type, int, int) {
    memcpy(out, in, (size_t)count * shim_mpi_size(type));
    return 0;
}
#endif
