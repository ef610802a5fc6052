/* Checkpoint and resume of device-resident trains in the reference's core
 * file format (paratt.c:1621-1892, pattac_write_tt_folder /
 * pattac_load_tt_folder): one file per core, <folder>/core_<k+1>.cr, header
 * "r_l,N,r_r\n", then the r_l*N*r_r values "%+1.16e\n" in column-major
 * order.  Seventeen significant digits round-trip every double exactly.
 *
 * ptt_checkpoint_begin queues the copy of the cores into page-locked host
 * memory on the train's stream and returns; a background thread waits for
 * the copy and writes the files (write-behind), so later work on the stream
 * neither waits for the disk nor changes the snapshot. */
#include <errno.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <cuda_runtime.h>

#include "paratt_b200.h"

struct ptt_checkpoint {
    pthread_t thread;
    int started;
    int device;
    cudaEvent_t done;          /* the copies have landed */
    double* host;              /* page-locked snapshot of the cores */
    int d, n[PTT_MAX_DIM], r[PTT_MAX_DIM + 1];
    char folder[4096];
    int status;                /* PTT_OK or a PTT_ERR_* code */
    char msg[4400];
};

static void* writer(void* arg) {
    struct ptt_checkpoint* cp = (struct ptt_checkpoint*)arg;
    cudaSetDevice(cp->device);
    if (cudaEventSynchronize(cp->done) != cudaSuccess) {
        cp->status = PTT_ERR_CUDA;
        snprintf(cp->msg, sizeof(cp->msg), "checkpoint: copy to the host failed");
        return NULL;
    }
    struct stat st;
    if (stat(cp->folder, &st) == -1 && mkdir(cp->folder, 0777) != 0 && errno != EEXIST) {
        cp->status = PTT_ERR_ARG;
        snprintf(cp->msg, sizeof(cp->msg), "checkpoint: can't create %s", cp->folder);
        return NULL;
    }
    const double* p = cp->host;
    char name[4200];
    for (int k = 0; k < cp->d; k++) {
        snprintf(name, sizeof(name), "%s/core_%d.cr", cp->folder, k + 1);
        FILE* fp = fopen(name, "w");
        if (!fp) {
            cp->status = PTT_ERR_ARG;
            snprintf(cp->msg, sizeof(cp->msg), "checkpoint: can't open %s", name);
            return NULL;
        }
        const size_t cnt = (size_t)cp->r[k] * cp->n[k] * cp->r[k + 1];
        fprintf(fp, "%d,%d,%d\n", cp->r[k], cp->n[k], cp->r[k + 1]);
        for (size_t e = 0; e < cnt; e++) fprintf(fp, "%+1.16e\n", p[e]);
        if (fclose(fp) != 0) {
            cp->status = PTT_ERR_ARG;
            snprintf(cp->msg, sizeof(cp->msg), "checkpoint: write to %s failed", name);
            return NULL;
        }
        p += cnt;
    }
    return NULL;
}

ptt_checkpoint* ptt_checkpoint_begin(ptt_tt* t, const char* folder) {
    if (!t || !folder || strlen(folder) >= 4096) return NULL;
    int d = 0;
    int n[PTT_MAX_DIM], cap[PTT_MAX_DIM + 1], r[PTT_MAX_DIM + 1];
    if (ptt_tt_shape(t, &d, n, cap)) return NULL;
    if (ptt_tt_get_ranks(t, r)) return NULL;
    double* dev[PTT_MAX_DIM];
    int* dr = NULL;
    if (ptt_tt_device_cores(t, dev, &dr)) return NULL;
    struct ptt_checkpoint* cp = (struct ptt_checkpoint*)calloc(1, sizeof(*cp));
    if (!cp) return NULL;
    cudaGetDevice(&cp->device);
    cp->d = d;
    memcpy(cp->n, n, sizeof(int) * d);
    memcpy(cp->r, r, sizeof(int) * (d + 1));
    snprintf(cp->folder, sizeof(cp->folder), "%s", folder);
    size_t total = 0;
    for (int k = 0; k < d; k++) total += (size_t)r[k] * n[k] * r[k + 1];
    cudaStream_t s = (cudaStream_t)ptt_ctx_stream(ptt_tt_context(t));
    if (cudaMallocHost((void**)&cp->host, sizeof(double) * (total ? total : 1)) != cudaSuccess ||
        cudaEventCreateWithFlags(&cp->done, cudaEventDisableTiming) != cudaSuccess) {
        cudaFreeHost(cp->host);
        free(cp);
        return NULL;
    }
    size_t off = 0;
    for (int k = 0; k < d; k++) {
        const size_t cnt = (size_t)r[k] * n[k] * r[k + 1];
        if (cudaMemcpyAsync(cp->host + off, dev[k], sizeof(double) * cnt, cudaMemcpyDeviceToHost, s) != cudaSuccess)
            cp->status = PTT_ERR_CUDA;
        off += cnt;
    }
    if (cudaEventRecord(cp->done, s) != cudaSuccess) cp->status = PTT_ERR_CUDA;
    if (cp->status == PTT_OK) {
        if (pthread_create(&cp->thread, NULL, writer, cp) == 0)
            cp->started = 1;
        else
            cp->status = PTT_ERR_ARG;
    }
    return cp;
}

int ptt_checkpoint_wait(ptt_checkpoint* cp) {
    if (!cp) return PTT_ERR_ARG;
    if (cp->started) pthread_join(cp->thread, NULL);
    const int st = cp->status;
    if (st && cp->msg[0]) fprintf(stderr, "paratt_b200: %s\n", cp->msg);
    cudaEventDestroy(cp->done);
    cudaFreeHost(cp->host);
    free(cp);
    return st;
}

/* one core file: header, then the values */
static int read_core(const char* name, int* rl, int* nn, int* rr, double** vals) {
    FILE* fp = fopen(name, "r");
    if (!fp) return PTT_ERR_ARG;
    if (fscanf(fp, "%d,%d,%d", rl, nn, rr) != 3 || *rl < 1 || *nn < 1 || *rr < 1) {
        fclose(fp);
        return PTT_ERR_ARG;
    }
    const size_t cnt = (size_t)(*rl) * (*nn) * (*rr);
    double* v = (double*)malloc(sizeof(double) * cnt);
    if (!v) {
        fclose(fp);
        return PTT_ERR_ARG;
    }
    for (size_t e = 0; e < cnt; e++)
        if (fscanf(fp, "%lf", &v[e]) != 1) {
            free(v);
            fclose(fp);
            return PTT_ERR_ARG;
        }
    fclose(fp);
    *vals = v;
    return PTT_OK;
}

int ptt_tt_load_folder(ptt_tt* t, const char* folder) {
    if (!t || !folder) return PTT_ERR_ARG;
    int d = 0;
    int n[PTT_MAX_DIM], cap[PTT_MAX_DIM + 1], r[PTT_MAX_DIM + 1];
    if (ptt_tt_shape(t, &d, n, cap)) return PTT_ERR_ARG;
    double* cores[PTT_MAX_DIM] = {0};
    char name[4200];
    int rc = PTT_OK;
    r[0] = 1;
    for (int k = 0; k < d && rc == PTT_OK; k++) {
        int rl, nn, rr;
        snprintf(name, sizeof(name), "%s/core_%d.cr", folder, k + 1);
        rc = read_core(name, &rl, &nn, &rr, &cores[k]);
        if (rc == PTT_OK && (nn != n[k] || rl != r[k] || (k == d - 1 && rr != 1))) {
            fprintf(stderr, "paratt_b200: %s: shape %d,%d,%d does not continue the train\n", name, rl, nn, rr);
            rc = PTT_ERR_ARG;
        }
        if (rc == PTT_OK) r[k + 1] = rr;
        else if (!cores[k]) fprintf(stderr, "paratt_b200: can't read %s\n", name);
    }
    if (rc == PTT_OK) rc = ptt_tt_set(t, r, (const double* const*)cores);
    for (int k = 0; k < d; k++) free(cores[k]);
    return rc;
}
