// Batched rounding of independent tensor trains (no counterpart in the
// reference, whose drivers round one train at a time).
//
// One rounding is a chain of small latency-bound launches that occupies a
// few SMs; independent trains are therefore rounded concurrently on worker
// contexts ("lanes": own stream, workspaces and tree counters, the parent's
// status word).  All ranks are read once up front, so issuing never waits
// for the device; trains go to the least-loaded lane, largest first (cost
// estimate sum_k r_k n_k r_{k+1} max(r_k, r_{k+1})), and the parent stream
// waits for every lane at the end, so later work on the parent context sees
// the rounded trains.
#include "ptt_common.cuh"

#include <stdlib.h>
#include <string.h>

static int lane_ctx(ptt_ctx* c, int i, ptt_ctx** out) {
    while (c->nlanes <= i) {
        ptt_ctx* l = ptt_ctx_create(c->device);
        if (!l) return ptt_last_error() ? ptt_last_error() : PTT_ERR_CUDA;
        cudaFree(l->d_status);
        l->d_status = c->d_status;
        l->shared_status = 1;
        l->lane = 1;
        c->lanes[c->nlanes++] = l;
    }
    c->lanes[i]->no_cholqr = c->no_cholqr;
    // no programmatic dependent launch on the lanes: a dependent grid's CTAs
    // occupy SMs while they wait for their predecessor, which on concurrent
    // lanes takes those SMs from the other lanes' ready kernels
    c->lanes[i]->no_pdl = 1;
    memcpy(c->lanes[i]->cq_cs, c->cq_cs, sizeof(c->cq_cs));
    c->lanes[i]->cq_tuned = c->cq_tuned;
    *out = c->lanes[i];
    return PTT_OK;
}

extern "C" int ptt_round_batch(ptt_tt* const* xs, int count, const double* tol, const int* const* maxrank,
                               int lanes) {
    if (count < 0 || (count > 0 && (!xs || !tol))) return ptt_set_error(PTT_ERR_ARG, "ptt_round_batch: bad arguments");
    if (count == 0) return PTT_OK;
    ptt_ctx* c = xs[0] ? xs[0]->ctx : NULL;
    for (int i = 0; i < count; i++) {
        if (!xs[i] || xs[i]->ctx != c) return ptt_set_error(PTT_ERR_ARG, "ptt_round_batch: trains must share one context");
        for (int j = 0; j < i; j++)
            if (xs[j] == xs[i]) return ptt_set_error(PTT_ERR_ARG, "ptt_round_batch: train %d repeated", i);
        if (!(tol[i] >= 0.0)) return ptt_set_error(PTT_ERR_ARG, "ptt_round_batch: tol[%d] must be >= 0", i);
    }
    if (lanes < 1) lanes = 1;
    if (lanes > PTT_MAX_LANES) lanes = PTT_MAX_LANES;
    if (lanes > count) lanes = count;
    PTT_CUDA(cudaSetDevice(c->device));
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    const int R = PTT_MAX_DIM + 1;
    int* rk = (int*)malloc(sizeof(int) * (size_t)R * count);
    double* cost = (double*)malloc(sizeof(double) * count);
    int* order = (int*)malloc(sizeof(int) * count);
    double load[PTT_MAX_LANES] = {0};
    int used[PTT_MAX_LANES] = {0};
    int rc = (rk && cost && order) ? PTT_OK : ptt_set_error(PTT_ERR_ARG, "ptt_round_batch: host allocation");
    for (int i = 0; i < count && !rc; i++) {
        int* r = rk + (size_t)R * i;
        rc = ptt_tt_get_ranks(xs[i], r);
        cost[i] = 0.0;
        for (int k = 0; k < xs[i]->d && !rc; k++) {
            const double rm = r[k] > r[k + 1] ? r[k] : r[k + 1];
            cost[i] += (double)r[k] * xs[i]->n[k] * r[k + 1] * rm;
        }
        order[i] = i;
    }
    // largest first (insertion sort: counts are small)
    for (int i = 1; i < count; i++)
        for (int j = i; j > 0 && cost[order[j]] > cost[order[j - 1]]; j--) {
            const int t = order[j];
            order[j] = order[j - 1];
            order[j - 1] = t;
        }
    for (int a = 0; a < count && !rc; a++) {
        const int i = order[a];
        int best = 0;
        for (int l = 1; l < lanes; l++)
            if (load[l] < load[best]) best = l;
        ptt_ctx* L;
        if ((rc = lane_ctx(c, best, &L))) break;
        xs[i]->ctx = L;
        rc = ptt_round_phases_rk(xs[i], rk + (size_t)R * i, tol[i], maxrank ? maxrank[i] : NULL, 3, 0);
        xs[i]->ctx = c;
        load[best] += cost[i];
        used[best] = 1;
    }
    for (int l = 0; l < lanes && l < c->nlanes; l++) {
        if (!used[l]) continue;
        ptt_ctx* L = c->lanes[l];
        cudaError_t e = cudaEventRecord(L->ev_join, L->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, L->ev_join, 0);
        if (e != cudaSuccess && !rc) rc = ptt_cuda_check(e, "ptt_round_batch join");
        c->launches += L->launches;
        L->launches = 0;
    }
    free(rk);
    free(cost);
    free(order);
    return rc;
}
