/* Test-only single-process stand-in for <mpi.h>.
 *
 * Part of the oracle (test infrastructure).  The reference simulator
 * (src/makefile:2 builds it with mpiCC) includes <mpi.h> from its runner
 * headers even when no MPI qubits are configured.  No MPI library is
 * installed here, so the oracle build puts this header on the include path.
 * Every MPI path in the reference is guarded by env.is_MPI (mpi_qbit > 0,
 * src/simulator.cpp:148), which the oracle never enables; these definitions
 * only have to compile and behave as a one-rank world.
 */
#ifndef QK_ORACLE_STUB_MPI_H
#define QK_ORACLE_STUB_MPI_H
#include <stdlib.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE_COMPLEX 0
#define MPI_THREAD_MULTIPLE 3
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

static inline int MPI_Init_thread(int *, char ***, int, int *provided) { if (provided) *provided = MPI_THREAD_MULTIPLE; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code); return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { abort(); return 0; }
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { abort(); return 0; }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { abort(); return 0; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { abort(); return 0; }
static inline int MPI_Sendrecv(const void *, int, MPI_Datatype, int, int, void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { abort(); return 0; }
#endif
