/* QUICK's C bridge (src/cuda/gpu.cu) compiled as host code for the oracle. */
#include "qref_shim.h"
#include "gpu.cu"

/* Read-back of the bridge's private state, for comparing QUICK's pair list
   and shell sort with this package's. */
extern "C" int qref_pairlist(int* xy, int cap, int* fStart, int* ffStart)
{
    int n = gpu->gpu_sim.sqrQshell;
    for (int i = 0; i < n && i < cap; i++) {
        xy[2 * i] = gpu->gpu_sim.sorted_YCutoffIJ[i].x;
        xy[2 * i + 1] = gpu->gpu_sim.sorted_YCutoffIJ[i].y;
    }
    *fStart = gpu->gpu_sim.fStart;
    *ffStart = gpu->gpu_sim.ffStart;
    return n;
}

extern "C" int qref_sorted_q(int* q, int* qnum, int cap)
{
    int n = gpu->gpu_sim.Qshell;
    for (int i = 0; i < n && i < cap; i++) {
        q[i] = gpu->gpu_sim.sorted_Q[i];
        qnum[i] = gpu->gpu_sim.sorted_Qnumber[i];
    }
    return n;
}

/* Prepare a fresh bridge object (gpu_startup_ leaves the POD members
   uninitialised, which QUICK's spdf bookkeeping then reads). */
extern "C" void qref_reset(void)
{
    gpu = new gpu_type();
    gpu->gpu_dev_id = -1;
}
