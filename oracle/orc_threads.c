/* orc_threads.c -- TEST INFRASTRUCTURE: thread control for the oracle. */
#include <omp.h>
void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int orc_get_threads(void) { return omp_get_max_threads(); }
