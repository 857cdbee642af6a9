/* GPU availability probe.  Replaces include/gpu/gpu.h:8 of the reference
 * (int gpu_backend_available(void)); returns 1 when a CUDA device of compute
 * capability 10.x is visible, 0 otherwise. */
#ifndef HPRQP_GPU_H
#define HPRQP_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

int gpu_backend_available(void);

#ifdef __cplusplus
}
#endif

#endif
