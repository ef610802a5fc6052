// Sketch-rank proposer: a 2-hidden-layer MLP (in -> W -> W -> 1, ReLU)
// with BF16 weights and FP32 accumulation, trained on the device with
// hand-written forward, backward and Adam kernels.
//
// Input per bond: the previous step's top-16 singular values of that bond as
// log10(sigma_j / delta) (delta = the bond's truncation threshold), the bond
// position k/d and the time step; output: the rank the bond needs in the
// next step's roundings, from which the sketch rank is taken.
//
// Parameters live in FP32 ("master", updated by Adam); the forward pass reads
// BF16 copies refreshed after every update, so gradients are those of the
// BF16-weight network with respect to its weights.
// Loss: mean of a (y - t)^2, a = under (y < t) or 1 (y >= t): predicting too
// few ranks costs a fallback, too many only a larger sketch.
#include "ptt_common.cuh"

#include <cuda_bf16.h>
#include <stdlib.h>
#include <string.h>

#define MLP_MAXW 128
#define MLP_MAXIN 64

struct ptt_mlp {
    ptt_ctx* ctx;
    int nin, w;
    long long np;          // number of parameters
    float* p;              // master parameters (device)
    __nv_bfloat16* pb;     // BF16 copies (device)
    float* g;              // gradients (device)
    float *m, *v;          // Adam moments
    long long t;           // Adam step
    float* x;              // staging for inputs / targets / outputs (device)
    float* tg;
    float* y;
    float* loss;
    int cap;               // batch capacity of the staging buffers
    float under;           // loss weight of under-prediction
};

// layout: W1 [w x nin], b1 [w], W2 [w x w], b2 [w], W3 [w], b3 [1]
static inline long long off_W1(int, int) { return 0; }
static inline long long off_b1(int nin, int w) { return (long long)w * nin; }
static inline long long off_W2(int nin, int w) { return off_b1(nin, w) + w; }
static inline long long off_b2(int nin, int w) { return off_W2(nin, w) + (long long)w * w; }
static inline long long off_W3(int nin, int w) { return off_b2(nin, w) + w; }
static inline long long off_b3(int nin, int w) { return off_W3(nin, w) + w; }
static inline long long mlp_np(int nin, int w) { return off_b3(nin, w) + 1; }

struct MlpDims {
    int nin, w;
    long long oW1, ob1, oW2, ob2, oW3, ob3;
};

static MlpDims dims_of(const ptt_mlp* m) {
    MlpDims d;
    d.nin = m->nin;
    d.w = m->w;
    d.oW1 = off_W1(m->nin, m->w);
    d.ob1 = off_b1(m->nin, m->w);
    d.oW2 = off_W2(m->nin, m->w);
    d.ob2 = off_b2(m->nin, m->w);
    d.oW3 = off_W3(m->nin, m->w);
    d.ob3 = off_b3(m->nin, m->w);
    return d;
}

// One sample per warp-iteration; weights staged in shared memory as FP32
// values of the BF16 copies.  Writes y; with grad != null also accumulates
// the gradients of the weighted squared error against tg.
__global__ void __launch_bounds__(256) k_mlp(MlpDims D, const __nv_bfloat16* pb, const float* p, const float* x,
                                             const float* tg, float* y, float* grad, float* loss, int B, float under) {
    extern __shared__ float sm[];
    const int nin = D.nin, w = D.w;
    float* W1 = sm;                 // w * nin
    float* b1 = W1 + w * nin;       // w
    float* W2 = b1 + w;             // w * w
    float* b2 = W2 + w * w;         // w
    float* W3 = b2 + w;             // w
    float* hb = W3 + w;             // per-warp scratch: 3 * w per warp
    const int np = (int)(D.ob3 + 1);
    for (int i = threadIdx.x; i < np - 1; i += blockDim.x) {
        float v;
        if (i < D.ob1)
            v = __bfloat162float(pb[D.oW1 + i]);
        else if (i < D.oW2)
            v = p[i];  // biases stay FP32
        else if (i < D.ob2)
            v = __bfloat162float(pb[i]);
        else if (i < D.oW3)
            v = p[i];
        else
            v = __bfloat162float(pb[i]);
        sm[i] = v;
    }
    __syncthreads();
    const float b3 = p[D.ob3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float* h1 = hb + warp * 3 * w;
    float* h2 = h1 + w;
    float* gh = h2 + w;
    float gloss = 0.f;
    for (int s = blockIdx.x * nw + warp; s < B; s += gridDim.x * nw) {
        const float* xs = x + (long long)s * nin;
        for (int o = lane; o < w; o += 32) {
            float a = b1[o];
            for (int i = 0; i < nin; i++) a = fmaf(W1[o * nin + i], xs[i], a);
            h1[o] = a > 0.f ? a : 0.f;
        }
        __syncwarp();
        for (int o = lane; o < w; o += 32) {
            float a = b2[o];
            for (int i = 0; i < w; i++) a = fmaf(W2[o * w + i], h1[i], a);
            h2[o] = a > 0.f ? a : 0.f;
        }
        __syncwarp();
        float a = 0.f;
        for (int i = lane; i < w; i += 32) a = fmaf(W3[i], h2[i], a);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        const float out = a + b3;
        if (lane == 0) y[s] = out;
        if (grad) {
            const float diff = out - tg[s];
            const float wt = diff < 0.f ? under : 1.f;
            gloss += wt * diff * diff;
            const float dy = 2.f * wt * diff / (float)B;
            // layer 3
            for (int i = lane; i < w; i += 32) atomicAdd(&grad[D.oW3 + i], dy * h2[i]);
            if (lane == 0) atomicAdd(&grad[D.ob3], dy);
            // dh2 = dy W3 * relu'(h2)
            for (int i = lane; i < w; i += 32) gh[i] = h2[i] > 0.f ? dy * W3[i] : 0.f;
            __syncwarp();
            for (int o = lane; o < w; o += 32) {
                const float go = gh[o];
                if (go != 0.f) {
                    for (int i = 0; i < w; i++) atomicAdd(&grad[D.oW2 + (long long)o * w + i], go * h1[i]);
                    atomicAdd(&grad[D.ob2 + o], go);
                }
            }
            // dh1 = W2^T dh2 * relu'(h1); reuse h2 as its storage
            __syncwarp();
            for (int i = lane; i < w; i += 32) {
                float acc = 0.f;
                for (int o = 0; o < w; o++) acc = fmaf(W2[o * w + i], gh[o], acc);
                h2[i] = h1[i] > 0.f ? acc : 0.f;
            }
            __syncwarp();
            for (int o = lane; o < w; o += 32) {
                const float go = h2[o];
                if (go != 0.f) {
                    for (int i = 0; i < nin; i++) atomicAdd(&grad[D.oW1 + (long long)o * nin + i], go * xs[i]);
                    atomicAdd(&grad[D.ob1 + o], go);
                }
            }
        }
        __syncwarp();
    }
    if (grad && lane == 0) atomicAdd(loss, gloss / (float)B);
}

__global__ void k_mlp_adam(float* p, __nv_bfloat16* pb, const float* g, float* m, float* v, long long np, float lr,
                           float b1, float b2, float eps, float c1, float c2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        pb[i] = __float2bfloat16_rn(pi);
    }
}

__global__ void k_mlp_refresh(const float* p, __nv_bfloat16* pb, long long np) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (long long)gridDim.x * blockDim.x)
        pb[i] = __float2bfloat16_rn(p[i]);
}

static size_t mlp_smem(const ptt_mlp* m) {
    return sizeof(float) * ((size_t)m->w * m->nin + 3 * (size_t)m->w + (size_t)m->w * m->w + 8 * 3 * (size_t)m->w);
}

static int stage(ptt_mlp* m, int B) {
    if (B <= m->cap) return PTT_OK;
    cudaFree(m->x);
    cudaFree(m->tg);
    cudaFree(m->y);
    m->x = m->tg = m->y = NULL;
    m->cap = 0;
    PTT_CUDA(cudaMalloc(&m->x, sizeof(float) * (size_t)B * m->nin));
    PTT_CUDA(cudaMalloc(&m->tg, sizeof(float) * (size_t)B));
    PTT_CUDA(cudaMalloc(&m->y, sizeof(float) * (size_t)B));
    m->cap = B;
    return PTT_OK;
}

extern "C" ptt_mlp* ptt_mlp_create(ptt_ctx* ctx, int nin, int width, unsigned long long seed) {
    if (!ctx || nin < 1 || nin > MLP_MAXIN || width < 1 || width > MLP_MAXW) {
        ptt_set_error(PTT_ERR_ARG, "ptt_mlp_create: bad sizes");
        return NULL;
    }
    ptt_mlp* m = (ptt_mlp*)calloc(1, sizeof(ptt_mlp));
    m->ctx = ctx;
    m->nin = nin;
    m->w = width;
    m->np = mlp_np(nin, width);
    m->under = 4.f;
    const size_t nb = sizeof(float) * (size_t)m->np;
    if (ptt_cuda_check(cudaMalloc(&m->p, nb), "mlp") || ptt_cuda_check(cudaMalloc(&m->g, nb), "mlp") ||
        ptt_cuda_check(cudaMalloc(&m->m, nb), "mlp") || ptt_cuda_check(cudaMalloc(&m->v, nb), "mlp") ||
        ptt_cuda_check(cudaMalloc(&m->pb, sizeof(__nv_bfloat16) * (size_t)m->np), "mlp") ||
        ptt_cuda_check(cudaMalloc(&m->loss, sizeof(float)), "mlp")) {
        free(m);
        return NULL;
    }
    // He-style initialisation from a host generator (splitmix64 + Box-Muller)
    float* h = (float*)malloc(nb);
    unsigned long long s = seed ? seed : 1;
    auto next = [&]() {
        s += 0x9E3779B97F4A7C15ull;
        unsigned long long z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return (double)((z ^ (z >> 31)) >> 11) * 1.1102230246251565e-16;
    };
    const MlpDims D = dims_of(m);
    for (long long i = 0; i < m->np; i++) {
        double u1 = next(), u2 = next();
        double g = sqrt(-2.0 * log(u1 + 1e-300)) * cos(6.283185307179586 * u2);
        double sc = 0.0;
        if (i < D.ob1)
            sc = sqrt(2.0 / nin);
        else if (i >= D.oW2 && i < D.ob2)
            sc = sqrt(2.0 / width);
        else if (i >= D.oW3 && i < D.ob3)
            sc = sqrt(1.0 / width);
        h[i] = (float)(g * sc);
    }
    cudaMemcpy(m->p, h, nb, cudaMemcpyHostToDevice);
    free(h);
    cudaMemset(m->m, 0, nb);
    cudaMemset(m->v, 0, nb);
    k_mlp_refresh<<<64, 256, 0, ctx->stream>>>(m->p, m->pb, m->np);
    ctx->launches++;
    if (ptt_cuda_check(cudaStreamSynchronize(ctx->stream), "mlp init")) {
        ptt_mlp_destroy(m);
        return NULL;
    }
    return m;
}

extern "C" void ptt_mlp_destroy(ptt_mlp* m) {
    if (!m) return;
    cudaStreamSynchronize(m->ctx->stream);
    cudaFree(m->p);
    cudaFree(m->pb);
    cudaFree(m->g);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->x);
    cudaFree(m->tg);
    cudaFree(m->y);
    cudaFree(m->loss);
    free(m);
}

extern "C" long long ptt_mlp_num_params(const ptt_mlp* m) { return m ? m->np : 0; }

extern "C" int ptt_mlp_get_params(ptt_mlp* m, float* out) {
    if (!m || !out) return ptt_set_error(PTT_ERR_ARG, "bad arguments");
    PTT_CUDA(cudaStreamSynchronize(m->ctx->stream));
    PTT_CUDA(cudaMemcpy(out, m->p, sizeof(float) * (size_t)m->np, cudaMemcpyDeviceToHost));
    return PTT_OK;
}

extern "C" int ptt_mlp_set_params(ptt_mlp* m, const float* in) {
    if (!m || !in) return ptt_set_error(PTT_ERR_ARG, "bad arguments");
    PTT_CUDA(cudaStreamSynchronize(m->ctx->stream));
    PTT_CUDA(cudaMemcpy(m->p, in, sizeof(float) * (size_t)m->np, cudaMemcpyHostToDevice));
    k_mlp_refresh<<<64, 256, 0, m->ctx->stream>>>(m->p, m->pb, m->np);
    PTT_LAUNCHED(m->ctx);
    PTT_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return PTT_OK;
}

static int run(ptt_mlp* m, const float* x, const float* t, int B, float* y, int want_grad) {
    if (!m || !x || B < 1) return ptt_set_error(PTT_ERR_ARG, "ptt_mlp: bad arguments");
    ptt_ctx* c = m->ctx;
    int rc = stage(m, B);
    if (rc) return rc;
    PTT_CUDA(cudaMemcpyAsync(m->x, x, sizeof(float) * (size_t)B * m->nin, cudaMemcpyHostToDevice, c->stream));
    if (want_grad) {
        PTT_CUDA(cudaMemcpyAsync(m->tg, t, sizeof(float) * (size_t)B, cudaMemcpyHostToDevice, c->stream));
        PTT_CUDA(cudaMemsetAsync(m->g, 0, sizeof(float) * (size_t)m->np, c->stream));
        PTT_CUDA(cudaMemsetAsync(m->loss, 0, sizeof(float), c->stream));
    }
    const MlpDims D = dims_of(m);
    int blocks = (B + 7) / 8;
    if (blocks > 296) blocks = 296;
    k_mlp<<<blocks, 256, mlp_smem(m), c->stream>>>(D, m->pb, m->p, m->x, m->tg, m->y, want_grad ? m->g : NULL,
                                                   m->loss, B, m->under);
    PTT_LAUNCHED(c);
    if (y) PTT_CUDA(cudaMemcpyAsync(y, m->y, sizeof(float) * (size_t)B, cudaMemcpyDeviceToHost, c->stream));
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    return PTT_OK;
}

extern "C" int ptt_mlp_forward(ptt_mlp* m, const float* x, int B, float* y) { return run(m, x, NULL, B, y, 0); }

extern "C" int ptt_mlp_grads(ptt_mlp* m, const float* x, const float* t, int B, float* grads, float* loss) {
    int rc = run(m, x, t, B, NULL, 1);
    if (rc) return rc;
    if (grads) PTT_CUDA(cudaMemcpy(grads, m->g, sizeof(float) * (size_t)m->np, cudaMemcpyDeviceToHost));
    if (loss) PTT_CUDA(cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
    return PTT_OK;
}

extern "C" int ptt_mlp_train_step(ptt_mlp* m, const float* x, const float* t, int B, float lr, float* loss) {
    int rc = run(m, x, t, B, NULL, 1);
    if (rc) return rc;
    m->t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)m->t), c2 = 1.f - powf(b2, (float)m->t);
    k_mlp_adam<<<64, 256, 0, m->ctx->stream>>>(m->p, m->pb, m->g, m->m, m->v, m->np, lr, b1, b2, 1e-8f, c1, c2);
    PTT_LAUNCHED(m->ctx);
    if (loss) PTT_CUDA(cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
    return PTT_OK;
}

extern "C" int ptt_mlp_set_under_weight(ptt_mlp* m, float w) {
    if (!m || !(w > 0.f)) return ptt_set_error(PTT_ERR_ARG, "bad weight");
    m->under = w;
    return PTT_OK;
}
