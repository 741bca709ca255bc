/*
 * profile.c -- opt-in per-kernel-class timing with CUDA events.
 *
 * The reference has a stand-alone tracer (tools/trace.c) that users wire in
 * by hand; here the library itself can bracket every tile-step launch with a
 * pair of events on the stream the kernel is launched on and accumulate, per
 * kernel class, the launches, the device time and the algorithmic work
 * (flops or bytes) of those launches.  Disabled by default: no events are
 * recorded unless plasma_profile_enable(1) was called.
 */
#include "../internal.h"

#include <cuda_runtime_api.h>
#include <stdlib.h>
#include <string.h>

#define MAX_REC 65536

typedef struct {
    cudaEvent_t e0, e1;
    int kclass;
    double flops, bytes;
} rec_t;

static int prof_on = 0;
static rec_t *recs = NULL;
static int nrec = 0;
static int nalloc = 0;

static long long acc_launch[PLASMA_KCLASS_COUNT];
static double acc_ms[PLASMA_KCLASS_COUNT];
static double acc_flops[PLASMA_KCLASS_COUNT];
static double acc_bytes[PLASMA_KCLASS_COUNT];

static void drain(void)
{
    for (int i = 0; i < nrec; i++) {
        float ms = 0.f;
        cudaEventSynchronize(recs[i].e1);
        cudaEventElapsedTime(&ms, recs[i].e0, recs[i].e1);
        int k = recs[i].kclass;
        acc_launch[k]++;
        acc_ms[k] += ms;
        acc_flops[k] += recs[i].flops;
        acc_bytes[k] += recs[i].bytes;
    }
    nrec = 0;
}

void plasma_profile_enable(int on)
{
    if (recs) drain();
    memset(acc_launch, 0, sizeof(acc_launch));
    memset(acc_ms, 0, sizeof(acc_ms));
    memset(acc_flops, 0, sizeof(acc_flops));
    memset(acc_bytes, 0, sizeof(acc_bytes));
    prof_on = on;
}

int plasma_profile_query(int kclass, long long *launches, double *ms,
                         double *flops, double *bytes)
{
    if (kclass < 0 || kclass >= PLASMA_KCLASS_COUNT)
        return PlasmaErrorIllegalValue;
    drain();
    if (launches) *launches = acc_launch[kclass];
    if (ms) *ms = acc_ms[kclass];
    if (flops) *flops = acc_flops[kclass];
    if (bytes) *bytes = acc_bytes[kclass];
    return PlasmaSuccess;
}

int plasma_prof_begin(cudaStream_t s)
{
    if (!prof_on)
        return -1;
    if (nrec >= MAX_REC)
        drain();
    if (nrec >= nalloc) {
        int grow = nalloc ? nalloc * 2 : 1024;
        if (grow > MAX_REC) grow = MAX_REC;
        recs = (rec_t *)realloc(recs, sizeof(rec_t) * grow);
        for (int i = nalloc; i < grow; i++) {
            cudaEventCreate(&recs[i].e0);
            cudaEventCreate(&recs[i].e1);
        }
        nalloc = grow;
    }
    int slot = nrec++;
    cudaEventRecord(recs[slot].e0, s);
    return slot;
}

void plasma_prof_end(int slot, cudaStream_t s, int kclass, double flops,
                     double bytes)
{
    if (slot < 0)
        return;
    recs[slot].kclass = kclass;
    recs[slot].flops = flops;
    recs[slot].bytes = bytes;
    cudaEventRecord(recs[slot].e1, s);
}
