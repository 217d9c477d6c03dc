/* The reference pair bodies are driven by the oracle's own host loop. */
#ifndef ORACLE_STUB_OMP_H
#define ORACLE_STUB_OMP_H
static inline int omp_get_thread_num(void) { return 0; }
static inline int omp_get_num_threads(void) { return 1; }
static inline int omp_get_max_threads(void) { return 1; }
#endif
