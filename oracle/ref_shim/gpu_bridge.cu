/* QUICK's C bridge (src/cuda/gpu.cu) compiled by nvcc for the GPU, unchanged:
 * build_ref.py --gpu links it with QUICK's gpu_type.cu, gpu_get2e.cu and
 * gpu_getxc.cu into oracle/_ref/gpu/libquickref.so, QUICK's own CUDA path run
 * on the device as a timed baseline.  Test and measurement infrastructure,
 * never the product. */
#include "gpu.cu"

/* A fresh bridge object (gpu_startup_ leaves its POD members uninitialised),
   on the device the caller names (gpu_set_device_ semantics). */
extern "C" void qref_reset(void)
{
    gpu = new gpu_type();
    gpu->gpu_dev_id = -1;
}
