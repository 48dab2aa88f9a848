/*
 * Test infrastructure (oracle) -- never product code.
 *
 * Functions of the reference's other modules that dump.c and restart.c name
 * (the AMR, boundary, GPU and grid paths); the writers ref_dumpio.c runs call
 * none of them. Kept apart from ref_dumpio.c, which includes the reference's
 * declarations: only the symbol names matter for the link.
 */
#include <stdlib.h>

void AMR_coord_linear2(void) { abort(); }
void GPU_boundprim(void) { abort(); }
void GPU_write(void) { abort(); }
void GPU_write_metric(void) { abort(); }
void bound_prim(void) { abort(); }
double divb_calc(void) { abort(); }
void set_grid(void) { abort(); }
int gpuDeviceSynchronize(void) { return 0; }
int gpuMemcpyAsync(void) { abort(); }
