/*
 * Host stand-in for the reference's src/statistics.cuh.  The original holds
 * two statistics kernels and their <<<>>> launches (ha_extfrag,
 * src/statistics.cuh:14-69); they are not on the malloc/free path and cannot
 * compile as host code, so the oracle build leaves them out.  ha_init()
 * records the pool split in two of that file's symbols
 * (src/halloc.cu:288-289), so those two stay, as plain host variables.
 */
static uint64 total_mem_g;
static uint64 cuda_mem_g;
