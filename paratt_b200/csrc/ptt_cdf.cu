// CDF-problem stencils and marginals of the reference (paratt.c:772-1618)
// with one process, on the device.
//
//  cdf_stencil       pattac_apply_cdf_stencil  paratt.c:772-923
//  cdf_lf_flux       pattac_apply_cdf_lf_flux  paratt.c:926-1093
//  cdf_lw_rhs        pattac_apply_cdf_lw_rhs   paratt.c:1096-1250
//  marginal_cusum    pattac_marginal_cusum     paratt.c:1393-1445
//  marginal_trap     pattac_marginal_trap      paratt.c:1448-1524
//  scale_weight_sum  pattac_scale_weight_sum   paratt.c:1527-1618
//  apply_marginal    pattac_apply_marginal     paratt.c:1252-1390
//
// With one process the reference's ghost cells are rows of the same core
// (its MPI exchange never runs), so every routine but the marginal is a scan
// along the mode index of each fiber core[i, :, k]: one thread per fiber,
// consecutive threads on consecutive i (coalesced), the result written to the
// core's second buffer and swapped in.  The scans keep the reference's order
// of operations per output value.
#include "ptt_common.cuh"

namespace {

enum { OP_STENCIL = 0, OP_LF = 1, OP_LW = 2, OP_CUSUM = 3, OP_TRAP = 4, OP_SWS = 5 };

// coefficient vectors in device memory: v0 [n or n+1] v1 v2 v3 (meaning per op)
struct ScanArgs {
    const double* v0;
    const double* v1;
    const double* v2;
    const double* v3;
    double s[16];  // stencil taps (OP_STENCIL)
    int slen;
    double dt, dx;
};

__global__ void k_fiber_scan(DevDesc* X, int k, int op, ScanArgs a) {
    const int r = X->r[k], n = X->n[k], r1 = X->r[k + 1];
    const long long nf = (long long)r * r1;
    const double* in = X->core[k];
    double* out = X->alt[k];
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < nf;
         f += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(f % r), kk = (int)(f / r);
        const double* x = in + i + (long long)r * n * kk;  // x[j * r]
        double* y = out + i + (long long)r * n * kk;
        const long long st = r;
        if (op == OP_STENCIL) {
            // ghost reads of the reference: j < 0 -> x[a - j - 1], j >= n -> x[2n - 1 - j]
            const int h = (a.slen - 1) / 2;
            for (int c = 0; c < n; c++) {
                double acc = 0.0;
                for (int t = 0; t < a.slen; t++) {
                    const int j = c - h + t;
                    const int src = j < 0 ? c - j - 1 : (j >= n ? 2 * n - 1 - j : j);
                    acc += a.s[t] * x[src * st];
                }
                y[c * st] = acc;
            }
        } else if (op == OP_LF) {
            // v0 = wave speed [n], v1 = ghost wave speeds [2], v2 = source [n]
            const double s0 = -0.5 / a.dx, s2 = 0.5 / a.dx;
            for (int c = 0; c < n; c++) {
                const double left = c - 1 < 0 ? -a.v1[0] * x[0] : -a.v0[c - 1] * x[(c - 1) * st];
                const double right = c + 1 >= n ? -a.v1[1] * x[(n - 1) * st] : -a.v0[c + 1] * x[(c + 1) * st];
                double acc = 0.0;
                acc += s0 * left;
                acc += s2 * right;
                y[c * st] = acc + a.v2[c] * x[c * st];
            }
        } else if (op == OP_LW) {
            // v0 = wave speed [n], v1 = ghost wave speeds [2], v2 = boundary
            // wave speeds [n + 1], v3 = source [n]
            const double g0 = x[0], g1 = x[(n - 1) * st];
            const double d2 = 2.0 * a.dx;
            double uh0 = 0.5 * (g0 + x[0]) - (a.v0[0] * x[0] - g0 * a.v1[0]) * a.dt / d2;
            for (int c = 0; c < n; c++) {
                const double xc = x[c * st];
                double uh1;
                if (c + 1 < n) {
                    const double xn = x[(c + 1) * st];
                    uh1 = 0.5 * (xn + xc) - (a.v0[c + 1] * xn - a.v0[c] * xc) * a.dt / d2;
                } else {
                    uh1 = 0.5 * (g1 + xc) - (g1 * a.v1[1] - a.v0[c] * xc) * a.dt / d2;
                }
                y[c * st] = -(a.v2[c + 1] * uh1 - a.v2[c] * uh0) / a.dx + a.v3[c] * xc;
                uh0 = uh1;
            }
        } else if (op == OP_CUSUM) {
            double cum = 0.0;
            for (int c = 0; c < n; c++) {
                const double v = x[c * st] * a.v0[c];
                cum = c == 0 ? v : cum + v;
                y[c * st] = cum;
            }
        } else {  // OP_TRAP, OP_SWS: trapezoid cumulative integral (weights v0)
            // OP_SWS adds scale[c] x[c] (scale in v1)
            double cum = 0.0, prev = x[0];
            for (int c = 1; c < n; c++) {
                const double cur = x[c * st];
                const double delta = 0.5 * a.v0[c] * (prev + cur);
                y[(c - 1) * st] = (op == OP_SWS) ? cum + prev * a.v1[c - 1] : cum;
                cum += delta;
                prev = cur;
            }
            y[(n - 1) * st] = (op == OP_SWS) ? cum + prev * a.v1[n - 1] : cum;
        }
    }
}

// W[p, q] = sum_j w[j] x_k[p, j, q]
__global__ void k_marg_w(const DevDesc* X, int k, const double* w, double* W) {
    const int r = X->r[k], n = X->n[k], r1 = X->r[k + 1];
    const double* x = X->core[k];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < r * r1; e += gridDim.x * blockDim.x) {
        const int p = e % r, q = e / r;
        double acc = 0.0;
        for (int j = 0; j < n; j++) acc += w[j] * x[p + (long long)r * (j + (long long)n * q)];
        W[e] = acc;
    }
}

// Z (d - 1 modes) from X with mode k contracted by W: cores before k copied,
// core k of Z = W x_{k+1} (k < d-1) or core k-1 of Z = x_{k-1} W (k = d-1),
// the cores after shifted down by one.  Grid y = core of Z.
// rank t of Z (d entries): X's ranks with r_{k+1} removed (k < d-1), or with
// r_{d-1} replaced by 1 (k = d-1), as pattac_apply_marginal allocates it
// (paratt.c:1263-1282)
__device__ __forceinline__ int marg_rank(const DevDesc* X, int k, int t) {
    const int d = X->d;
    if (k < d - 1) return t <= k ? X->r[t] : X->r[t + 1];
    return t < d - 1 ? X->r[t] : 1;
}

__global__ void k_marg_build(const DevDesc* X, int k, const double* W, DevDesc* Z, int* status) {
    const int d = X->d;
    const int kz = blockIdx.y;
    if (kz >= d - 1) return;
    const int src = (kz < k) ? kz : kz + 1;  // X core copied into Z core kz
    const bool fold_next = (k < d - 1 && kz == k);
    const bool fold_prev = (k == d - 1 && kz == k - 1);
    const int rz = marg_rank(X, k, kz), rz1 = marg_rank(X, k, kz + 1);
    const int nz = X->n[src];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Z->r[kz] = rz;
        if (kz == d - 2) Z->r[d - 1] = 1;
    }
    const long long cnt = (long long)rz * nz * rz1;
    if (rz > Z->rcap[kz] || rz1 > Z->rcap[kz + 1] || cnt > Z->cap[kz] || Z->n[kz] != nz) {
        if (blockIdx.x == 0 && threadIdx.x == 0) PTT_STATUS_SET(status, PTT_ERR_CAPACITY);
        return;
    }
    double* z = Z->core[kz];
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long e0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (fold_next) {  // z[p, jc] = sum_q W[p, q] x_{k+1}[q, jc]
        const int r1 = X->r[k + 1];
        const double* xn = X->core[k + 1];
        for (long long e = e0; e < cnt; e += stride) {
            const int p = (int)(e % rz);
            const long long jc = e / rz;
            double acc = 0.0;
            for (int q = 0; q < r1; q++) acc += W[p + (long long)rz * q] * xn[q + (long long)r1 * jc];
            z[e] = acc;
        }
    } else if (fold_prev) {  // z[i] = sum_q x_{k-1}[i + m q] W[q], m = r_{k-1} n_{k-1}
        const int rq = X->r[k];
        const long long m = (long long)X->r[k - 1] * X->n[k - 1];
        const double* xp = X->core[k - 1];
        for (long long e = e0; e < cnt; e += stride) {
            double acc = 0.0;
            for (int q = 0; q < rq; q++) acc += W[q] * xp[e + m * q];
            z[e] = acc;
        }
    } else {
        const double* xs = X->core[src];
        for (long long e = e0; e < cnt; e += stride) z[e] = xs[e];
    }
}

int scan_launch(ptt_tt* x, int mode, int op, ScanArgs& a, const double* const* host, const int* lens, int nvec) {
    if (!x || mode < 0 || mode >= x->d) return ptt_set_error(PTT_ERR_ARG, "bad train or mode");
    ptt_ctx* c = x->ctx;
    size_t tot = 0;
    for (int v = 0; v < nvec; v++) tot += (size_t)lens[v];
    int rc = ptt_ws_reserve(c, sizeof(double) * (tot + 8) + 256);
    if (rc) return rc;
    double* dv = (double*)c->ws;
    const double** slots[4] = {&a.v0, &a.v1, &a.v2, &a.v3};
    size_t off = 0;
    for (int v = 0; v < nvec; v++) {
        if (!host[v]) return ptt_set_error(PTT_ERR_ARG, "null coefficient vector");
        PTT_CUDA(cudaMemcpyAsync(dv + off, host[v], sizeof(double) * lens[v], cudaMemcpyHostToDevice, c->stream));
        *slots[v] = dv + off;
        off += (size_t)lens[v];
    }
    const long long nf = (long long)x->rcap[mode] * x->rcap[mode + 1];
    long long bx = (nf + 127) / 128;
    if (bx > 8LL * c->nsm) bx = 8LL * c->nsm;
    if (bx < 1) bx = 1;
    k_fiber_scan<<<(unsigned)bx, 128, 0, c->stream>>>(x->dd, mode, op, a);
    PTT_LAUNCHED(c);
    // host copies are done when the stream passes this point; the caller's
    // vectors may be reused once the call returns (synchronous copies above)
    return ptt_swap(x, mode, mode + 1);
}

}  // namespace

extern "C" int ptt_cdf_stencil(ptt_tt* x, int mode, const double* sten, int slen) {
    ScanArgs a = {};
    if (!sten) return ptt_set_error(PTT_ERR_ARG, "ptt_cdf_stencil: null stencil");
    if (slen % 2 == 0) slen -= 1;  // paratt.c:786: even lengths drop the last tap
    if (slen < 1 || slen > 15) return ptt_set_error(PTT_ERR_ARG, "ptt_cdf_stencil: stencil length %d", slen);
    if (x && mode >= 0 && mode < x->d && (slen - 1) / 2 > x->n[mode])
        return ptt_set_error(PTT_ERR_ARG, "ptt_cdf_stencil: half-width exceeds the mode size");
    for (int t = 0; t < slen; t++) a.s[t] = sten[t];
    a.slen = slen;
    return scan_launch(x, mode, OP_STENCIL, a, nullptr, nullptr, 0);
}

extern "C" int ptt_cdf_lf_flux(ptt_tt* x, int mode, const double* wave_speed, const double* gc_wave_speed,
                               const double* source_coef, double dt, double dx) {
    if (!x || mode < 0 || mode >= x->d) return ptt_set_error(PTT_ERR_ARG, "ptt_cdf_lf_flux: bad train or mode");
    ScanArgs a = {};
    a.dt = dt;
    a.dx = dx;
    const int n = x->n[mode];
    const double* h[3] = {wave_speed, gc_wave_speed, source_coef};
    const int l[3] = {n, 2, n};
    return scan_launch(x, mode, OP_LF, a, h, l, 3);
}

extern "C" int ptt_cdf_lw_rhs(ptt_tt* x, int mode, const double* wave_speed, const double* gc_wave_speed,
                              const double* bdry_wave_speed, const double* source_coef, double dt, double dx) {
    if (!x || mode < 0 || mode >= x->d) return ptt_set_error(PTT_ERR_ARG, "ptt_cdf_lw_rhs: bad train or mode");
    ScanArgs a = {};
    a.dt = dt;
    a.dx = dx;
    const int n = x->n[mode];
    const double* h[4] = {wave_speed, gc_wave_speed, bdry_wave_speed, source_coef};
    const int l[4] = {n, 2, n + 1, n};
    return scan_launch(x, mode, OP_LW, a, h, l, 4);
}

extern "C" int ptt_marginal_cusum(ptt_tt* x, int mode, const double* w) {
    if (!x || mode < 0 || mode >= x->d) return ptt_set_error(PTT_ERR_ARG, "ptt_marginal_cusum: bad train or mode");
    ScanArgs a = {};
    const double* h[1] = {w};
    const int l[1] = {x->n[mode]};
    return scan_launch(x, mode, OP_CUSUM, a, h, l, 1);
}

extern "C" int ptt_marginal_trap(ptt_tt* x, int mode, const double* w) {
    if (!x || mode < 0 || mode >= x->d) return ptt_set_error(PTT_ERR_ARG, "ptt_marginal_trap: bad train or mode");
    ScanArgs a = {};
    const double* h[1] = {w};
    const int l[1] = {x->n[mode]};
    return scan_launch(x, mode, OP_TRAP, a, h, l, 1);
}

extern "C" int ptt_scale_weight_sum(ptt_tt* x, int mode, const double* scale, const double* sum_w) {
    if (!x || mode < 0 || mode >= x->d) return ptt_set_error(PTT_ERR_ARG, "ptt_scale_weight_sum: bad train or mode");
    ScanArgs a = {};
    const double* h[2] = {sum_w, scale};
    const int l[2] = {x->n[mode], x->n[mode]};
    return scan_launch(x, mode, OP_SWS, a, h, l, 2);
}

extern "C" int ptt_apply_marginal(const ptt_tt* x, int mode, const double* w, ptt_tt* z) {
    if (!x || !z || !w || mode < 0 || mode >= x->d || x->d < 2 || z->d != x->d - 1)
        return ptt_set_error(PTT_ERR_ARG, "ptt_apply_marginal: bad arguments (z needs d - 1 modes)");
    for (int k = 0; k < z->d; k++)
        if (z->n[k] != x->n[k < mode ? k : k + 1])
            return ptt_set_error(PTT_ERR_ARG, "ptt_apply_marginal: mode %d of z does not match", k);
    ptt_ctx* c = x->ctx;
    if (z->ctx != c) return ptt_set_error(PTT_ERR_ARG, "ptt_apply_marginal: trains of different contexts");
    const int n = x->n[mode];
    const long long wsz = (long long)x->rcap[mode] * x->rcap[mode + 1];
    int rc = ptt_ws_reserve(c, sizeof(double) * (size_t)(n + wsz + 8) + 256);
    if (rc) return rc;
    double* dw = (double*)c->ws;
    double* W = dw + n;
    PTT_CUDA(cudaMemcpyAsync(dw, w, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    int bx = (int)((wsz + 255) / 256);
    if (bx > 1024) bx = 1024;
    k_marg_w<<<bx < 1 ? 1 : bx, 256, 0, c->stream>>>(x->dd, mode, dw, W);
    PTT_LAUNCHED(c);
    long long mx = 1;
    for (int k = 0; k < z->d; k++) mx = z->cap[k] > mx ? z->cap[k] : mx;
    long long gx = (mx + 255) / 256;
    const int cap = ptt_core_grid_cap(c, z->d);
    if (gx > cap) gx = cap;
    k_marg_build<<<dim3((unsigned)gx, z->d), 256, 0, c->stream>>>(x->dd, mode, W, z->dd, c->d_status);
    PTT_LAUNCHED(c);
    return PTT_OK;
}
