// fsb_select.cu -- the learned plan selector's device side: matrix features
// of a CSR structure, and the forward / backward / Adam kernels of the
// selector's multilayer perceptron.
//
// The network is small (16 inputs, two hidden layers of 64 ReLU units, one
// output per candidate plan, at most 32), trained on a few thousand samples:
// its layers are 64-wide matrix-vector products, far below the size where
// tensor-core tiles pay, so these are plain FMA kernels.  Every reduction
// runs in a fixed order, so training is deterministic run to run.
//
// Parameter layout (float32, one contiguous buffer):
//   W1[d_in][h1], b1[h1], W2[h1][h2], b2[h2], W3[h2][d_out], b3[d_out]
// Activation cache per sample: Z1[h1], Z2[h2] (pre-activations), Y[d_out].
#include "fsb_dispatch.cuh"

namespace fsb {

constexpr int kMlpMaxIn = 16;
constexpr int kMlpMaxHidden = 64;
constexpr int kMlpMaxOut = 32;

// ----------------------------------------------------------- features ----
// Per-matrix sums over rows / nonzeros: out[0] = sum of row lengths,
// out[1] = sum of squared row lengths, out[2] = longest row, out[3] = empty
// rows, out[4] = sum over nonzeros of |col - r * n_cols / n_rows| / n_cols
// (distance from the scaled diagonal).  out must hold zeros on entry.
template <class I, class P>
__global__ void __launch_bounds__(256) k_csr_features(const P* __restrict__ ptr, const I* __restrict__ col,
                                                      int64_t n_rows, int64_t n_cols, double* __restrict__ out) {
    __shared__ double s_sum[8], s_sq[8], s_band[8], s_empty[8], s_aligned[8];
    __shared__ unsigned long long s_max[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double sum = 0, sq = 0, band = 0, empty = 0, aligned = 0;
    unsigned long long mx = 0;
    const double scale = n_rows > 0 ? (double)n_cols / (double)n_rows : 0.0;
    const double inv_cols = n_cols > 0 ? 1.0 / (double)n_cols : 0.0;
    for (int64_t r = (int64_t)blockIdx.x * 8 + warp; r < n_rows; r += (int64_t)gridDim.x * 8) {
        const int64_t s = idx(ptr[r]), e = idx(ptr[r + 1]);
        const double len = (double)(e - s);
        if (lane == 0) {
            sum += len;
            sq += len * len;
            empty += (e == s) ? 1.0 : 0.0;
            if ((unsigned long long)(e - s) > mx) mx = (unsigned long long)(e - s);
        }
        const double diag = (double)r * scale;
        for (int64_t k = s + lane; k < e; k += 32) {
            const int64_t c = idx(col[k]);
            band += fabs((double)c - diag) * inv_cols;
            // in a row of aligned dense 16-column blocks, column and position
            // in the row agree modulo 16
            aligned += ((c & 15) == ((k - s) & 15)) ? 1.0 : 0.0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        band += __shfl_xor_sync(0xffffffffu, band, o);
        aligned += __shfl_xor_sync(0xffffffffu, aligned, o);
    }
    if (lane == 0) {
        s_sum[warp] = sum;
        s_sq[warp] = sq;
        s_band[warp] = band;
        s_empty[warp] = empty;
        s_aligned[warp] = aligned;
        s_max[warp] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, c = 0, d = 0, al = 0;
        unsigned long long m = 0;
        for (int w = 0; w < 8; ++w) {
            a += s_sum[w];
            b += s_sq[w];
            c += s_band[w];
            d += s_empty[w];
            al += s_aligned[w];
            m = s_max[w] > m ? s_max[w] : m;
        }
        atomicAdd(out + 0, a);
        atomicAdd(out + 1, b);
        atomicMax(reinterpret_cast<unsigned long long*>(out + 2), m);  // integer held in the slot's bits
        atomicAdd(out + 3, d);
        atomicAdd(out + 4, c);
        atomicAdd(out + 5, al);
    }
}

// ---------------------------------------------------------------- MLP ----
struct MlpDims {
    int d_in, h1, h2, d_out;
};

__device__ __forceinline__ int mlp_off_b1(const MlpDims& m) { return m.d_in * m.h1; }
__device__ __forceinline__ int mlp_off_w2(const MlpDims& m) { return m.d_in * m.h1 + m.h1; }
__device__ __forceinline__ int mlp_off_b2(const MlpDims& m) { return mlp_off_w2(m) + m.h1 * m.h2; }
__device__ __forceinline__ int mlp_off_w3(const MlpDims& m) { return mlp_off_b2(m) + m.h2; }
__device__ __forceinline__ int mlp_off_b3(const MlpDims& m) { return mlp_off_w3(m) + m.h2 * m.d_out; }
static int mlp_param_count(const MlpDims& m) {
    return m.d_in * m.h1 + m.h1 + m.h1 * m.h2 + m.h2 + m.h2 * m.d_out + m.d_out;
}

// Forward: one warp per sample; the parameters are staged in shared memory.
// cache (optional) receives Z1, Z2 and Y per sample.
__global__ void __launch_bounds__(256) k_mlp_forward(const float* __restrict__ X, int n, const float* __restrict__ prm,
                                                     MlpDims m, float* __restrict__ Y, float* __restrict__ cache) {
    extern __shared__ float sp[];
    const int np = m.d_in * m.h1 + m.h1 + m.h1 * m.h2 + m.h2 + m.h2 * m.d_out + m.d_out;
    for (int i = threadIdx.x; i < np; i += blockDim.x) sp[i] = prm[i];
    __shared__ float sx[8][kMlpMaxIn], sh1[8][kMlpMaxHidden], sh2[8][kMlpMaxHidden];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float* W1 = sp;
    const float* b1 = sp + mlp_off_b1(m);
    const float* W2 = sp + mlp_off_w2(m);
    const float* b2 = sp + mlp_off_b2(m);
    const float* W3 = sp + mlp_off_w3(m);
    const float* b3 = sp + mlp_off_b3(m);
    const int cstride = m.h1 + m.h2 + m.d_out;
    for (int s = blockIdx.x * 8 + warp; s < n; s += gridDim.x * 8) {
        if (lane < m.d_in) sx[warp][lane] = X[(int64_t)s * m.d_in + lane];
        __syncwarp();
        for (int j = lane; j < m.h1; j += 32) {
            float z = b1[j];
            for (int i = 0; i < m.d_in; ++i) z = fmaf(sx[warp][i], W1[i * m.h1 + j], z);
            sh1[warp][j] = z > 0.f ? z : 0.f;
            if (cache) cache[(int64_t)s * cstride + j] = z;
        }
        __syncwarp();
        for (int j = lane; j < m.h2; j += 32) {
            float z = b2[j];
            for (int i = 0; i < m.h1; ++i) z = fmaf(sh1[warp][i], W2[i * m.h2 + j], z);
            sh2[warp][j] = z > 0.f ? z : 0.f;
            if (cache) cache[(int64_t)s * cstride + m.h1 + j] = z;
        }
        __syncwarp();
        for (int k = lane; k < m.d_out; k += 32) {
            float y = b3[k];
            for (int i = 0; i < m.h2; ++i) y = fmaf(sh2[warp][i], W3[i * m.d_out + k], y);
            Y[(int64_t)s * m.d_out + k] = y;
            if (cache) cache[(int64_t)s * cstride + m.h1 + m.h2 + k] = y;
        }
        __syncwarp();
    }
}

// Backward, step 1 (one warp per sample): masked squared-error loss against
// T, output delta dY = 2 (Y - T) mask / n_terms, and the hidden deltas
// dZ2 = (dY W3^T) * [Z2 > 0], dZ1 = (dZ2 W2^T) * [Z1 > 0].
// deltas per sample: dZ1[h1], dZ2[h2], dY[d_out]; loss_terms[s] = sum of the
// sample's masked squared errors.
__global__ void __launch_bounds__(256) k_mlp_deltas(const float* __restrict__ cache, const float* __restrict__ T,
                                                    const float* __restrict__ mask, int n, float inv_terms,
                                                    const float* __restrict__ prm, MlpDims m,
                                                    float* __restrict__ deltas, float* __restrict__ loss_terms) {
    __shared__ float sdy[8][kMlpMaxOut], sdz2[8][kMlpMaxHidden];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float* W2 = prm + mlp_off_w2(m);
    const float* W3 = prm + mlp_off_w3(m);
    const int cstride = m.h1 + m.h2 + m.d_out;
    for (int s = blockIdx.x * 8 + warp; s < n; s += gridDim.x * 8) {
        const float* c = cache + (int64_t)s * cstride;
        float* d = deltas + (int64_t)s * cstride;
        float l = 0.f;
        for (int k = lane; k < m.d_out; k += 32) {
            const float mk = mask[(int64_t)s * m.d_out + k];
            const float diff = c[m.h1 + m.h2 + k] - T[(int64_t)s * m.d_out + k];
            const float dy = 2.f * diff * mk * inv_terms;
            l += mk * diff * diff;
            sdy[warp][k] = dy;
            d[m.h1 + m.h2 + k] = dy;
        }
        for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
        if (lane == 0) loss_terms[s] = l;
        __syncwarp();
        for (int j = lane; j < m.h2; j += 32) {
            float g = 0.f;
            for (int k = 0; k < m.d_out; ++k) g = fmaf(sdy[warp][k], W3[j * m.d_out + k], g);
            g = c[m.h1 + j] > 0.f ? g : 0.f;
            sdz2[warp][j] = g;
            d[m.h1 + j] = g;
        }
        __syncwarp();
        for (int i = lane; i < m.h1; i += 32) {
            float g = 0.f;
            for (int j = 0; j < m.h2; ++j) g = fmaf(sdz2[warp][j], W2[i * m.h2 + j], g);
            d[i] = c[i] > 0.f ? g : 0.f;
        }
        __syncwarp();
    }
}

// Backward, step 2: one thread per parameter, summing over the samples in
// order (deterministic).  Layer inputs: X for layer 1, relu(Z1) for layer 2,
// relu(Z2) for layer 3.
__global__ void __launch_bounds__(256) k_mlp_grads(const float* __restrict__ X, const float* __restrict__ cache,
                                                   const float* __restrict__ deltas, int n, MlpDims m,
                                                   float* __restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int cstride = m.h1 + m.h2 + m.d_out;
    const int o_b1 = m.d_in * m.h1, o_w2 = o_b1 + m.h1, o_b2 = o_w2 + m.h1 * m.h2, o_w3 = o_b2 + m.h2,
              o_b3 = o_w3 + m.h2 * m.d_out, np = o_b3 + m.d_out;
    if (p >= np) return;
    float g = 0.f;
    if (p < o_b1) {  // W1[i][j]
        const int i = p / m.h1, j = p % m.h1;
        for (int s = 0; s < n; ++s) g = fmaf(X[(int64_t)s * m.d_in + i], deltas[(int64_t)s * cstride + j], g);
    } else if (p < o_w2) {  // b1[j]
        const int j = p - o_b1;
        for (int s = 0; s < n; ++s) g += deltas[(int64_t)s * cstride + j];
    } else if (p < o_b2) {  // W2[i][j]
        const int q = p - o_w2, i = q / m.h2, j = q % m.h2;
        for (int s = 0; s < n; ++s) {
            const float a = cache[(int64_t)s * cstride + i];
            g = fmaf(a > 0.f ? a : 0.f, deltas[(int64_t)s * cstride + m.h1 + j], g);
        }
    } else if (p < o_w3) {  // b2[j]
        const int j = p - o_b2;
        for (int s = 0; s < n; ++s) g += deltas[(int64_t)s * cstride + m.h1 + j];
    } else if (p < o_b3) {  // W3[i][k]
        const int q = p - o_w3, i = q / m.d_out, k = q % m.d_out;
        for (int s = 0; s < n; ++s) {
            const float a = cache[(int64_t)s * cstride + m.h1 + i];
            g = fmaf(a > 0.f ? a : 0.f, deltas[(int64_t)s * cstride + m.h1 + m.h2 + k], g);
        }
    } else {  // b3[k]
        const int k = p - o_b3;
        for (int s = 0; s < n; ++s) g += deltas[(int64_t)s * cstride + m.h1 + m.h2 + k];
    }
    grad[p] = g;
}

// Adam (Kingma & Ba 2015) with bias correction; step counts from 1.
__global__ void k_adam(float* __restrict__ prm, const float* __restrict__ grad, float* __restrict__ m1,
                       float* __restrict__ m2, int np, float lr, float beta1, float beta2, float eps, float bc1,
                       float bc2, float weight_decay) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const float g = grad[p] + weight_decay * prm[p];
    const float a = beta1 * m1[p] + (1.f - beta1) * g;
    const float b = beta2 * m2[p] + (1.f - beta2) * g * g;
    m1[p] = a;
    m2[p] = b;
    prm[p] -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
}

static int check_dims(const MlpDims& m) {
    if (m.d_in < 1 || m.d_in > kMlpMaxIn || m.h1 < 1 || m.h1 > kMlpMaxHidden || m.h2 < 1 || m.h2 > kMlpMaxHidden ||
        m.d_out < 1 || m.d_out > kMlpMaxOut) {
        fsb_host::set_error("mlp dims must be d_in <= %d, hidden <= %d, d_out <= %d", kMlpMaxIn, kMlpMaxHidden,
                            kMlpMaxOut);
        return FSB_ERR_INVALID;
    }
    return FSB_OK;
}

}  // namespace fsb

using fsb::MlpDims;

extern "C" int fsb_csr_features(const void* row_ptr, int ptr_dtype, const void* col_idx, int index_dtype,
                                int64_t n_rows, int64_t n_cols, double* out, void* stream) {
    if (!row_ptr || !out || n_rows < 0 || n_cols < 0) {
        fsb_host::set_error("fsb_csr_features: bad arguments");
        return FSB_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(out, 0, 5 * sizeof(double), st);
    if (e != cudaSuccess) {
        fsb_host::set_error("fsb_csr_features: %s", cudaGetErrorString(e));
        return FSB_ERR_LAUNCH;
    }
    if (n_rows == 0) return FSB_OK;
    return fsb::dispatch_idx(index_dtype, [&](auto ti) -> int {
        using I = typename decltype(ti)::type;
        return fsb::dispatch_idx(ptr_dtype, [&](auto tp) -> int {
            using P = typename decltype(tp)::type;
            int64_t blocks = fsb::ceil_div(n_rows, (int64_t)8);
            if (blocks > 148 * 16) blocks = 148 * 16;
            fsb::k_csr_features<I, P><<<(unsigned)blocks, 256, 0, st>>>(
                static_cast<const P*>(row_ptr), static_cast<const I*>(col_idx), n_rows, n_cols, out);
            return fsb_host::check_launch("k_csr_features");
        });
    });
}

extern "C" int fsb_mlp_param_count(int d_in, int h1, int h2, int d_out) {
    MlpDims m{d_in, h1, h2, d_out};
    if (fsb::check_dims(m)) return FSB_ERR_INVALID;
    return fsb::mlp_param_count(m);
}

extern "C" int fsb_mlp_forward(const float* X, int n, int d_in, int h1, int h2, int d_out, const float* params,
                               float* Y, float* cache, void* stream) {
    MlpDims m{d_in, h1, h2, d_out};
    if (int rc = fsb::check_dims(m)) return rc;
    if (n < 0 || (n > 0 && (!X || !params || !Y))) {
        fsb_host::set_error("fsb_mlp_forward: bad arguments");
        return FSB_ERR_INVALID;
    }
    if (n == 0) return FSB_OK;
    const size_t smem = (size_t)fsb::mlp_param_count(m) * sizeof(float);
    const int blocks = (int)fsb::ceil_div((int64_t)n, (int64_t)8) < 148 * 4 ? (int)fsb::ceil_div((int64_t)n, (int64_t)8)
                                                                           : 148 * 4;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(fsb::k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) {
            fsb_host::set_error("cudaFuncSetAttribute: %s", cudaGetErrorString(e));
            return FSB_ERR_LAUNCH;
        }
    }
    fsb::k_mlp_forward<<<blocks, 256, smem, st>>>(X, n, params, m, Y, cache);
    return fsb_host::check_launch("k_mlp_forward");
}

extern "C" int fsb_mlp_backward(const float* X, int n, int d_in, int h1, int h2, int d_out, const float* params,
                                const float* cache, const float* targets, const float* mask, float inv_terms,
                                float* deltas, float* loss_terms, float* grad, void* stream) {
    MlpDims m{d_in, h1, h2, d_out};
    if (int rc = fsb::check_dims(m)) return rc;
    if (n < 1 || !X || !params || !cache || !targets || !mask || !deltas || !loss_terms || !grad) {
        fsb_host::set_error("fsb_mlp_backward: bad arguments");
        return FSB_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int blocks = (int)fsb::ceil_div((int64_t)n, (int64_t)8) < 148 * 4 ? (int)fsb::ceil_div((int64_t)n, (int64_t)8)
                                                                           : 148 * 4;
    fsb::k_mlp_deltas<<<blocks, 256, 0, st>>>(cache, targets, mask, n, inv_terms, params, m, deltas, loss_terms);
    int rc = fsb_host::check_launch("k_mlp_deltas");
    if (rc) return rc;
    const int np = fsb::mlp_param_count(m);
    fsb::k_mlp_grads<<<(np + 255) / 256, 256, 0, st>>>(X, cache, deltas, n, m, grad);
    return fsb_host::check_launch("k_mlp_grads");
}

extern "C" int fsb_adam_step(float* params, const float* grad, float* m1, float* m2, int n_params, float lr,
                             float beta1, float beta2, float eps, int step, float weight_decay, void* stream) {
    if (!params || !grad || !m1 || !m2 || n_params < 1 || step < 1) {
        fsb_host::set_error("fsb_adam_step: bad arguments");
        return FSB_ERR_INVALID;
    }
    const float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
    fsb::k_adam<<<(n_params + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        params, grad, m1, m2, n_params, lr, beta1, beta2, eps, bc1, bc2, weight_decay);
    return fsb_host::check_launch("k_adam");
}
