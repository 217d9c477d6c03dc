/* Minimal single-process stand-in for the MPI declarations the reference's
 * headers name. Test infrastructure only: the reference pair bodies compiled
 * by oracle/build_ref.sh run in one process and never communicate. */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Group;
typedef int MPI_Win;
typedef int MPI_Info;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_INT 1
#define MPI_LONG 2
#define MPI_LONG_LONG 3
#define MPI_DOUBLE 4
#define MPI_FLOAT 5
#define MPI_BYTE 6
#define MPI_CHAR 7
#define MPI_UNSIGNED_LONG_LONG 8
#define MPI_UNSIGNED_LONG 9
#define MPI_UNSIGNED 10
#define MPI_SHORT 11
#define MPI_UNSIGNED_CHAR 12
#define MPI_LONG_LONG_INT 13
#define MPI_INT64_T 14
#define MPI_UINT64_T 15
#define MPI_UNSIGNED_SHORT 16
#define MPI_C_BOOL 17
#define MPI_CXX_BOOL 18
#define MPI_INT32_T 19
#define MPI_UINT32_T 20
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LOR 4
#define MPI_LAND 5
#define MPI_BOR 6
#define MPI_BAND 7
#define MPI_MAXLOC 8
#define MPI_MINLOC 9
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_SUCCESS 0
#define MPI_REQUEST_NULL 0
#define MPI_UNDEFINED (-32766)
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_DOUBLE_INT 21
#define MPI_2INT 22
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_MULTIPLE 3
static inline int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm, int) { return 0; }
#endif
