/*
 * oracle.c -- CPU restatement of FlagSparse's CSR/COO SpMV and SpMM path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the CPU oracle that the CUDA
 * kernels of flagsparse_public_b200 are tested against: it is used by tests/,
 * by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by the
 * library itself.
 *
 * What it restates (paths relative to the FlagSparse project root):
 *   orc_spmv_csr   : _spmv_csr_real_kernel / _spmv_csr_complex_kernel and the
 *                    CSR-vector bucket kernels (src/flagsparse/sparse_operations/
 *                    spmv_csr.py:158-343): y[r] = sum_k A[r,k] x[col[k]] over the
 *                    row's nonzeros (capped at row_cap when > 0, as the plain
 *                    kernel's MAX_SEGMENTS * BLOCK_NNZ window does, :175-183),
 *                    accumulated in the compute precision of the path:
 *                    acc_mode 0 (native) f16/bf16/f32 -> f32, f64 -> f64,
 *                    c64 -> f32 pairs (:246, :306); acc_mode 1 (wide) f32 -> f64,
 *                    c64 -> f64 pairs (:116-121, spmm_coo.py:11-18).
 *   orc_spmm_csr   : _spmm_csr_real_kernel and the opt / alg2 / COO row-run
 *                    kernels (spmm_csr.py:92-195, :602-919,
 *                    spmm_csr_opt_alg2.py:338-629, spmm_coo.py:135-241).
 *   orc_*_exact    : the FP64 oracle the error bounds of the tests are stated
 *                    against: products split exactly (TwoProduct by fma) and
 *                    summed with Neumaier's compensated summation in double, so
 *                    the result is the exact sum rounded (almost always) once.
 *   orc_csr_transpose   : _transpose_csr_for_spmv (spmv_csr.py:456-494), a
 *                         stable sort of the nonzeros by column.
 *   orc_coo_lex_order   : _sort_coo_lex_inplace (spmv_coo.py:297-309,
 *                         spmm_coo.py:21-32) and the sort of coo_to_csr_for_spmv
 *                         (spmv_csr.py:885-909), stable on (row, col).
 *   orc_seg_starts      : _seg_starts_from_sorted_rows (spmv_coo.py:312-327).
 *   orc_split_metadata  : _build_spmm_opt_split_metadata (spmm_csr.py:417-441).
 *   orc_sddmm_csr       : _sddmm_csr_real_kernel (sddmm_csr.py:108-152):
 *                         out[p] = alpha * dot(x[row(p)], y[col(p)]) +
 *                         beta * data[p], the dot product accumulated in the
 *                         value precision (float32 / float64) in K order.
 *   orc_spmm_diag       : the diagnose-only stable / candidate SpMM arithmetic
 *                         (spmm_csr.py:922-1249, :1501-1634): fixed-order
 *                         float64 or Kahan accumulation per element.
 *   orc_merge_partition : restatement of the merge-path partition kernel
 *                         (Merrill & Garland's merge-path search over row ends
 *                         and nonzero indices).
 *   orc_merge_runs      : the split-row runs of a partition (which units hold
 *                         parts of one row), by a linear walk -- the unit-level
 *                         form of the long-row split metadata above.
 *
 * Sums run in row order, one nonzero after the other; the reference's Triton
 * kernels sum 256-lane tiles as trees, so agreement is to rounding, not bits,
 * for floating point, and bit-exact for all integer structure.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_F16 0
#define ORC_BF16 1
#define ORC_F32 2
#define ORC_F64 3
#define ORC_C64 4
#define ORC_C128 5
#define ORC_I32 6
#define ORC_I64 7

/* ---------------------------------------------------- half conversions -- */
/* IEEE 754 binary16 / bfloat16 <-> binary32 by bit manipulation, round to
 * nearest even on narrowing. */
static float f16_to_f32(uint16_t h) {
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1fu;
    uint32_t man = h & 0x3ffu;
    uint32_t bits;
    if (exp == 0) {
        if (man == 0) {
            bits = sign;
        } else { /* subnormal: normalise */
            int e = -1;
            do { man <<= 1; ++e; } while (!(man & 0x400u));
            man &= 0x3ffu;
            bits = sign | ((uint32_t)(127 - 15 - e) << 23) | (man << 13);
        }
    } else if (exp == 0x1f) {
        bits = sign | 0x7f800000u | (man << 13);
    } else {
        bits = sign | ((exp + 127 - 15) << 23) | (man << 13);
    }
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

static uint16_t f32_to_f16(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) return (uint16_t)(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u : 0)); /* inf/nan */
    if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u); /* rounds to inf */
    if (ax < 0x38800000u) { /* subnormal or zero in half */
        if (ax < 0x33000000u) return (uint16_t)sign; /* < half of smallest subnormal */
        uint32_t e = ax >> 23;
        uint32_t m = (ax & 0x7fffffu) | 0x800000u;
        int shift = (int)(126 - e); /* 14 + (112 - e) + ... */
        /* value = m * 2^(e-150); half subnormal unit = 2^-24 -> q = m >> (126 - e) */
        uint32_t q = m >> shift;
        uint32_t rem = m & ((1u << shift) - 1u);
        uint32_t half = 1u << (shift - 1);
        if (rem > half || (rem == half && (q & 1u))) ++q;
        return (uint16_t)(sign | q);
    }
    uint32_t e = (ax >> 23) - 127 + 15;
    uint32_t m = ax & 0x7fffffu;
    uint32_t q = (e << 10) | (m >> 13);
    uint32_t rem = m & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) ++q;
    return (uint16_t)(sign | q);
}

static float bf16_to_f32(uint16_t h) {
    uint32_t bits = (uint32_t)h << 16;
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

static uint16_t f32_to_bf16(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    if ((x & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((x >> 16) | 0x40u); /* quiet nan */
    uint32_t lsb = (x >> 16) & 1u;
    x += 0x7fffu + lsb;
    return (uint16_t)(x >> 16);
}

/* ----------------------------------------------------------- accessors -- */
static inline int64_t ld_idx(const void* p, int dt, int64_t i) {
    return dt == ORC_I64 ? ((const int64_t*)p)[i] : (int64_t)((const int32_t*)p)[i];
}
/* Real value (or real part) as double: exact for every supported type. */
static inline double ld_re(const void* p, int dt, int64_t i) {
    switch (dt) {
    case ORC_F16: return (double)f16_to_f32(((const uint16_t*)p)[i]);
    case ORC_BF16: return (double)bf16_to_f32(((const uint16_t*)p)[i]);
    case ORC_F32: return (double)((const float*)p)[i];
    case ORC_F64: return ((const double*)p)[i];
    case ORC_C64: return (double)((const float*)p)[2 * i];
    case ORC_C128: return ((const double*)p)[2 * i];
    default: return 0.0;
    }
}
static inline double ld_im(const void* p, int dt, int64_t i) {
    switch (dt) {
    case ORC_C64: return (double)((const float*)p)[2 * i + 1];
    case ORC_C128: return ((const double*)p)[2 * i + 1];
    default: return 0.0;
    }
}
static inline int is_complex(int dt) { return dt == ORC_C64 || dt == ORC_C128; }

static void st_val(void* p, int dt, int64_t i, double re, double im) {
    switch (dt) {
    case ORC_F16: ((uint16_t*)p)[i] = f32_to_f16((float)re); break;
    case ORC_BF16: ((uint16_t*)p)[i] = f32_to_bf16((float)re); break;
    case ORC_F32: ((float*)p)[i] = (float)re; break;
    case ORC_F64: ((double*)p)[i] = re; break;
    case ORC_C64: ((float*)p)[2 * i] = (float)re; ((float*)p)[2 * i + 1] = (float)im; break;
    case ORC_C128: ((double*)p)[2 * i] = re; ((double*)p)[2 * i + 1] = im; break;
    default: break;
    }
}

/* Accumulation precision of (value dtype, acc mode): 1 = f32, 2 = f64. */
static int acc_prec(int vdt, int acc_mode) {
    if (vdt == ORC_F64 || vdt == ORC_C128) return 2;
    if (acc_mode == 1 && (vdt == ORC_F32 || vdt == ORC_C64)) return 2;
    return 1;
}

/* One dot product sum_k a_k * b_k in the path's precision; a_k from the
 * sparse values at index k, b_k from the dense operand at index bi(k). */
typedef struct { double re, im; } orc_c;

static orc_c dot_row(const void* val, int vdt, const void* col, int idt, int64_t s, int64_t e,
                     const void* dense, int64_t ld, int64_t c, int prec) {
    orc_c acc = {0.0, 0.0};
    if (!is_complex(vdt)) {
        if (prec == 1) {
            float a32 = 0.f;
            for (int64_t k = s; k < e; ++k) {
                const int64_t j = ld_idx(col, idt, k);
                a32 = fmaf((float)ld_re(val, vdt, k), (float)ld_re(dense, vdt, j * ld + c), a32);
            }
            acc.re = a32;
        } else {
            double a64 = 0.0;
            for (int64_t k = s; k < e; ++k) {
                const int64_t j = ld_idx(col, idt, k);
                a64 = fma(ld_re(val, vdt, k), ld_re(dense, vdt, j * ld + c), a64);
            }
            acc.re = a64;
        }
        return acc;
    }
    if (prec == 1) {
        float re = 0.f, im = 0.f;
        for (int64_t k = s; k < e; ++k) {
            const int64_t j = ld_idx(col, idt, k);
            const float ar = (float)ld_re(val, vdt, k), ai = (float)ld_im(val, vdt, k);
            const float br = (float)ld_re(dense, vdt, j * ld + c), bi = (float)ld_im(dense, vdt, j * ld + c);
            re = fmaf(ar, br, re);
            re = fmaf(-ai, bi, re);
            im = fmaf(ar, bi, im);
            im = fmaf(ai, br, im);
        }
        acc.re = re;
        acc.im = im;
    } else {
        double re = 0.0, im = 0.0;
        for (int64_t k = s; k < e; ++k) {
            const int64_t j = ld_idx(col, idt, k);
            const double ar = ld_re(val, vdt, k), ai = ld_im(val, vdt, k);
            const double br = ld_re(dense, vdt, j * ld + c), bi = ld_im(dense, vdt, j * ld + c);
            re = fma(ar, br, re);
            re = fma(-ai, bi, re);
            im = fma(ar, bi, im);
            im = fma(ai, br, im);
        }
        acc.re = re;
        acc.im = im;
    }
    return acc;
}

/* Fast path of the common case: f32 values, int32 columns. */
static void spmv_f32_i32(const float* val, const int32_t* col, const void* ptr, int pdt, int64_t n_rows,
                         const float* x, float* y, int prec, int64_t row_cap, int threads) {
#pragma omp parallel for schedule(dynamic, 1024) num_threads(threads)
    for (int64_t r = 0; r < n_rows; ++r) {
        const int64_t s = ld_idx(ptr, pdt, r);
        int64_t e = ld_idx(ptr, pdt, r + 1);
        if (row_cap > 0 && e - s > row_cap) e = s + row_cap;
        if (prec == 2) {
            double a = 0.0;
            for (int64_t k = s; k < e; ++k) a = fma((double)val[k], (double)x[col[k]], a);
            y[r] = (float)a;
        } else {
            float a = 0.f;
            for (int64_t k = s; k < e; ++k) a = fmaf(val[k], x[col[k]], a);
            y[r] = a;
        }
    }
}

static void spmm_f32_i32(const float* val, const int32_t* col, const void* ptr, int pdt, int64_t n_rows,
                         const float* B, int64_t ldb, int64_t n_dense, float* C, int64_t ldc, int prec,
                         int threads) {
#pragma omp parallel num_threads(threads)
    {
        double* acc = (double*)malloc(sizeof(double) * (size_t)(n_dense > 0 ? n_dense : 1));
        float* accf = (float*)malloc(sizeof(float) * (size_t)(n_dense > 0 ? n_dense : 1));
#pragma omp for schedule(dynamic, 256)
        for (int64_t r = 0; r < n_rows; ++r) {
            const int64_t s = ld_idx(ptr, pdt, r), e = ld_idx(ptr, pdt, r + 1);
            if (prec == 2) {
                for (int64_t c = 0; c < n_dense; ++c) acc[c] = 0.0;
                for (int64_t k = s; k < e; ++k) {
                    const double a = (double)val[k];
                    const float* b = B + (int64_t)col[k] * ldb;
                    for (int64_t c = 0; c < n_dense; ++c) acc[c] = fma(a, (double)b[c], acc[c]);
                }
                for (int64_t c = 0; c < n_dense; ++c) C[r * ldc + c] = (float)acc[c];
            } else {
                for (int64_t c = 0; c < n_dense; ++c) accf[c] = 0.f;
                for (int64_t k = s; k < e; ++k) {
                    const float a = val[k];
                    const float* b = B + (int64_t)col[k] * ldb;
                    for (int64_t c = 0; c < n_dense; ++c) accf[c] = fmaf(a, b[c], accf[c]);
                }
                for (int64_t c = 0; c < n_dense; ++c) C[r * ldc + c] = accf[c];
            }
        }
        free(acc);
        free(accf);
    }
}

/* y = A x.  out_dtype is the value dtype, or f32 for f16/bf16 values. */
int orc_spmv_csr(const void* val, const void* col, const void* ptr, int vdt, int idt, int pdt, int64_t n_rows,
                 const void* x, void* y, int out_dtype, int acc_mode, int64_t row_cap, int threads) {
    if (threads < 1) threads = 1;
    const int prec = acc_prec(vdt, acc_mode);
    if (vdt == ORC_F32 && idt == ORC_I32 && out_dtype == ORC_F32) {
        spmv_f32_i32((const float*)val, (const int32_t*)col, ptr, pdt, n_rows, (const float*)x, (float*)y, prec,
                     row_cap, threads);
        return 0;
    }
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads)
    for (int64_t r = 0; r < n_rows; ++r) {
        const int64_t s = ld_idx(ptr, pdt, r);
        int64_t e = ld_idx(ptr, pdt, r + 1);
        if (row_cap > 0 && e - s > row_cap) e = s + row_cap;
        orc_c a = dot_row(val, vdt, col, idt, s, e, x, 1, 0, prec);
        st_val(y, out_dtype, r, a.re, a.im);
    }
    return 0;
}

/* C = A B, B row-major n_cols x n_dense (stride ldb), C n_rows x n_dense (ldc). */
int orc_spmm_csr(const void* val, const void* col, const void* ptr, int vdt, int idt, int pdt, int64_t n_rows,
                 const void* B, int64_t ldb, int64_t n_dense, void* C, int64_t ldc, int out_dtype, int acc_mode,
                 int threads) {
    if (threads < 1) threads = 1;
    const int prec = acc_prec(vdt, acc_mode);
    if (vdt == ORC_F32 && idt == ORC_I32 && out_dtype == ORC_F32) {
        spmm_f32_i32((const float*)val, (const int32_t*)col, ptr, pdt, n_rows, (const float*)B, ldb, n_dense,
                     (float*)C, ldc, prec, threads);
        return 0;
    }
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t r = 0; r < n_rows; ++r) {
        const int64_t s = ld_idx(ptr, pdt, r), e = ld_idx(ptr, pdt, r + 1);
        for (int64_t c = 0; c < n_dense; ++c) {
            orc_c a = dot_row(val, vdt, col, idt, s, e, B, ldb, c, prec);
            st_val(C, out_dtype, r * ldc + c, a.re, a.im);
        }
    }
    return 0;
}

/* -------------------------------------------- diagnostic SpMM forms -- */
/* FlagSparse's diagnose-only SpMM arithmetic (spmm_csr.py:922-1249 stable
 * kernels, :1501-1634 candidate short-row kernels), per output element in
 * nonzero order: mode 0 acc = fma(a, b, acc) in the value precision; 1 the
 * same in double, stored in the value type; 2 Kahan in the value precision
 * (y = fma(a, b, -comp); t = acc + y; comp = (t - acc) - y; acc = t); 3 Kahan
 * in double.  Rows of at most short_max nonzeros use mode_short.  The
 * fused multiply-adds are written out (fma / fmaf) and the file is built
 * with -ffp-contract=off, so every operation is rounded where written. */
static double diag_dot_d(const void* val, int vdt, const void* col, int idt, int64_t s, int64_t e, const void* B,
                         int64_t ldb, int64_t n, int kahan) {
    double acc = 0.0, comp = 0.0;
    for (int64_t k = s; k < e; ++k) {
        const double a = ld_re(val, vdt, k), b = ld_re(B, vdt, ld_idx(col, idt, k) * ldb + n);
        if (kahan) {
            const double y = fma(a, b, -comp), t = acc + y;
            comp = (t - acc) - y;
            acc = t;
        } else {
            acc = fma(a, b, acc);
        }
    }
    return acc;
}

static float diag_dot_f(const float* val, const void* col, int idt, int64_t s, int64_t e, const float* B,
                        int64_t ldb, int64_t n, int kahan) {
    float acc = 0.f, comp = 0.f;
    for (int64_t k = s; k < e; ++k) {
        const float a = val[k], b = B[ld_idx(col, idt, k) * ldb + n];
        if (kahan) {
            const float y = fmaf(a, b, -comp), t = acc + y;
            comp = (t - acc) - y;
            acc = t;
        } else {
            acc = fmaf(a, b, acc);
        }
    }
    return acc;
}

int orc_spmm_diag(const void* val, const void* col, const void* ptr, int vdt, int idt, int pdt, int64_t n_rows,
                  const void* B, int64_t ldb, int64_t n_dense, void* C, int64_t ldc, int mode_short, int mode_long,
                  int64_t short_max, int threads) {
    if (vdt != ORC_F32 && vdt != ORC_F64) return -1;
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t r = 0; r < n_rows; ++r) {
        const int64_t s = ld_idx(ptr, pdt, r), e = ld_idx(ptr, pdt, r + 1);
        const int mode = (e - s) <= short_max ? mode_short : mode_long;
        const int kahan = mode == 2 || mode == 3;
        for (int64_t n = 0; n < n_dense; ++n) {
            if (vdt == ORC_F64 || mode == 1 || mode == 3) {
                const double v = diag_dot_d(val, vdt, col, idt, s, e, B, ldb, n, kahan);
                if (vdt == ORC_F64) ((double*)C)[r * ldc + n] = v;
                else ((float*)C)[r * ldc + n] = (float)v;
            } else {
                ((float*)C)[r * ldc + n] =
                    diag_dot_f((const float*)val, col, idt, s, e, (const float*)B, ldb, n, kahan);
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------- FP64 oracle -- */
/* Neumaier summation of exact products (TwoProduct by fma). */
typedef struct { double s, c; } orc_sum;
static inline void nsum_add(orc_sum* a, double v) {
    const double t = a->s + v;
    if (fabs(a->s) >= fabs(v)) a->c += (a->s - t) + v; else a->c += (v - t) + a->s;
    a->s = t;
}
static inline void nsum_prod(orc_sum* a, double x, double y) {
    const double p = x * y;
    nsum_add(a, p);
    nsum_add(a, fma(x, y, -p));
}

static void dot_exact(const void* val, int vdt, const void* col, int idt, int64_t s, int64_t e, const void* dense,
                      int64_t ld, int64_t c, double* re, double* im, double* abs_sum) {
    orc_sum sr = {0.0, 0.0}, si = {0.0, 0.0};
    double mag = 0.0;
    for (int64_t k = s; k < e; ++k) {
        const int64_t j = ld_idx(col, idt, k);
        const double ar = ld_re(val, vdt, k), br = ld_re(dense, vdt, j * ld + c);
        if (is_complex(vdt)) {
            const double ai = ld_im(val, vdt, k), bi = ld_im(dense, vdt, j * ld + c);
            nsum_prod(&sr, ar, br);
            nsum_prod(&sr, -ai, bi);
            nsum_prod(&si, ar, bi);
            nsum_prod(&si, ai, br);
            mag += hypot(ar, ai) * hypot(br, bi);
        } else {
            nsum_prod(&sr, ar, br);
            mag += fabs(ar * br);
        }
    }
    *re = sr.s + sr.c;
    *im = si.s + si.c;
    if (abs_sum) *abs_sum = mag;
}

/* y_re/y_im: double results; abs_sum: sum |a_k b_k| per row (condition scale). */
int orc_spmv_csr_exact(const void* val, const void* col, const void* ptr, int vdt, int idt, int pdt, int64_t n_rows,
                       const void* x, double* y_re, double* y_im, double* abs_sum, int threads) {
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads)
    for (int64_t r = 0; r < n_rows; ++r) {
        double re, im, mag;
        dot_exact(val, vdt, col, idt, ld_idx(ptr, pdt, r), ld_idx(ptr, pdt, r + 1), x, 1, 0, &re, &im, &mag);
        y_re[r] = re;
        if (y_im) y_im[r] = im;
        if (abs_sum) abs_sum[r] = mag;
    }
    return 0;
}

int orc_spmm_csr_exact(const void* val, const void* col, const void* ptr, int vdt, int idt, int pdt, int64_t n_rows,
                       const void* B, int64_t ldb, int64_t n_dense, double* c_re, double* c_im, double* abs_sum,
                       int threads) {
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t r = 0; r < n_rows; ++r) {
        const int64_t s = ld_idx(ptr, pdt, r), e = ld_idx(ptr, pdt, r + 1);
        for (int64_t c = 0; c < n_dense; ++c) {
            double re, im, mag;
            dot_exact(val, vdt, col, idt, s, e, B, ldb, c, &re, &im, &mag);
            c_re[r * n_dense + c] = re;
            if (c_im) c_im[r * n_dense + c] = im;
            if (abs_sum) abs_sum[r * n_dense + c] = mag;
        }
    }
    return 0;
}

/* --------------------------------------------------- integer structure -- */
/* Stable counting sort of the nonzeros by column: CSR of A^T.
 * t_ptr[n_cols+1], t_rows[nnz] (row id of each transposed entry),
 * perm[nnz] (source nonzero of each transposed entry). */
int orc_csr_transpose(const void* ptr, int pdt, const void* col, int idt, int64_t n_rows, int64_t n_cols,
                      int64_t nnz, int64_t* t_ptr, int64_t* t_rows, int64_t* perm) {
    memset(t_ptr, 0, sizeof(int64_t) * (size_t)(n_cols + 1));
    for (int64_t k = 0; k < nnz; ++k) t_ptr[ld_idx(col, idt, k) + 1]++;
    for (int64_t c = 0; c < n_cols; ++c) t_ptr[c + 1] += t_ptr[c];
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n_cols > 0 ? n_cols : 1));
    if (!fill) return -1;
    memcpy(fill, t_ptr, sizeof(int64_t) * (size_t)n_cols);
    for (int64_t r = 0; r < n_rows; ++r) {
        for (int64_t k = ld_idx(ptr, pdt, r); k < ld_idx(ptr, pdt, r + 1); ++k) {
            const int64_t c = ld_idx(col, idt, k);
            const int64_t dst = fill[c]++;
            t_rows[dst] = r;
            perm[dst] = k;
        }
    }
    free(fill);
    return 0;
}

/* Stable merge sort of nonzeros by key = row * max(1, n_cols) + col. */
static void msort(int64_t* idx, int64_t* tmp, const int64_t* key, int64_t n) {
    for (int64_t w = 1; w < n; w <<= 1) {
        for (int64_t lo = 0; lo < n; lo += 2 * w) {
            int64_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
            int64_t i = lo, j = mid, o = lo;
            while (i < mid && j < hi) tmp[o++] = key[idx[j]] < key[idx[i]] ? idx[j++] : idx[i++];
            while (i < mid) tmp[o++] = idx[i++];
            while (j < hi) tmp[o++] = idx[j++];
        }
        memcpy(idx, tmp, sizeof(int64_t) * (size_t)n);
    }
}

int orc_coo_lex_order(const int64_t* row, const int64_t* col, int64_t nnz, int64_t n_cols, int64_t* perm) {
    int64_t* key = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nnz > 0 ? nnz : 1));
    int64_t* tmp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nnz > 0 ? nnz : 1));
    if (!key || !tmp) return -1;
    const int64_t scale = n_cols > 1 ? n_cols : 1;
    for (int64_t k = 0; k < nnz; ++k) {
        key[k] = row[k] * scale + col[k];
        perm[k] = k;
    }
    msort(perm, tmp, key, nnz);
    free(key);
    free(tmp);
    return 0;
}

/* Row-run offsets of row-sorted COO; returns the number of runs. */
int64_t orc_seg_starts(const int64_t* row_sorted, int64_t nnz, int64_t* seg) {
    if (nnz == 0) return 0;
    int64_t n = 0;
    seg[n++] = 0;
    for (int64_t k = 1; k < nnz; ++k)
        if (row_sorted[k] != row_sorted[k - 1]) seg[n++] = k;
    seg[n] = nnz;
    return n;
}

/* Long-row split: parts of part_nnz nonzeros for each row id in long_rows. */
int64_t orc_split_metadata(const int64_t* indptr, const int64_t* long_rows, int64_t n_long, int64_t part_nnz,
                           int64_t* part_rows, int64_t* part_starts, int64_t* part_ends, int64_t* row_part_ptr) {
    int64_t n = 0;
    row_part_ptr[0] = 0;
    for (int64_t i = 0; i < n_long; ++i) {
        const int64_t r = long_rows[i];
        int64_t cur = indptr[r];
        const int64_t end = indptr[r + 1];
        while (cur < end) {
            part_rows[n] = r;
            part_starts[n] = cur;
            cur = cur + part_nnz < end ? cur + part_nnz : end;
            part_ends[n] = cur;
            ++n;
        }
        row_part_ptr[i + 1] = n;
    }
    return n;
}

/* Merge-path coordinates (rows ended, nonzeros consumed) of diagonals
 * u * items, u in [0, n_units]; interior boundaries inside rows shorter
 * than snap are moved back to the row start. */
int orc_merge_partition(const void* ptr, int pdt, int64_t n_rows, int64_t nnz, int64_t items, int64_t snap,
                        int64_t n_units, int64_t* coords) {
    const int64_t total = n_rows + nnz;
    for (int64_t u = 0; u <= n_units; ++u) {
        int64_t d = u * items;
        if (d > total) d = total;
        /* linear walk reference: count row ends r with ptr[r+1] <= d - (rows before) ... via search */
        int64_t lo = d - nnz > 0 ? d - nnz : 0, hi = d < n_rows ? d : n_rows;
        while (lo < hi) {
            const int64_t mid = (lo + hi) / 2;
            if (ld_idx(ptr, pdt, mid + 1) <= d - mid - 1) lo = mid + 1; else hi = mid;
        }
        int64_t i = lo, j = d - lo;
        if (snap > 0 && i < n_rows && u > 0 && u < n_units) {
            const int64_t rs = ld_idx(ptr, pdt, i), re = ld_idx(ptr, pdt, i + 1);
            if (j > rs && re - rs < snap) j = rs;
        }
        coords[2 * u] = i;
        coords[2 * u + 1] = j;
    }
    return 0;
}

/* Split-row runs of a merge-path partition, by a linear walk over the units:
 * unit u is open when its end (r, k) lies inside row r after r's start and
 * after u's own start; its run is the maximal sequence of consecutive units
 * open on row r, extended by the unit holding r's end.  runs[2u] / [2u + 1]
 * = first / last unit of that run, -1 for units that are not open.  (The
 * reference splits long rows on the host, spmm_csr.py:417-441; this is the
 * same bookkeeping for merge-path units.) */
int orc_merge_runs(const void* ptr, int pdt, int64_t n_rows, const int64_t* coords, int64_t n_units,
                   int64_t* runs) {
    for (int64_t u = 0; u < n_units; ++u) {
        runs[2 * u] = -1;
        runs[2 * u + 1] = -1;
    }
    int64_t u = 0;
    while (u < n_units) {
        const int64_t r = coords[2 * u + 2], k1 = coords[2 * u + 3], k0 = coords[2 * u + 1];
        int open = 0;
        if (r < n_rows) {
            const int64_t s = ld_idx(ptr, pdt, r);
            open = k1 > (s > k0 ? s : k0);
        }
        if (!open) {
            ++u;
            continue;
        }
        /* u opens a run on row r: every following unit that ends on row r
         * continues it, the first unit ending past row r closes it */
        int64_t v = u;
        while (v < n_units && coords[2 * v + 2] == r) ++v;
        /* v: first unit whose end row is past r (holds r's end) */
        for (int64_t w = u; w < v; ++w) {
            runs[2 * w] = u;
            runs[2 * w + 1] = v;
        }
        u = v;
    }
    return 0;
}

/* SDDMM on a CSR pattern (float32 or float64 values, vdt), rows in parallel. */
int orc_sddmm_csr(const void* col, int idt, const void* ptr, int pdt, int64_t n_rows, const void* x, int64_t ldx,
                  const void* y, int64_t ldy, int64_t k, const void* data, void* out, int vdt, double alpha,
                  double beta, int threads) {
    if (vdt != ORC_F32 && vdt != ORC_F64) return -2;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads)
    for (int64_t r = 0; r < n_rows; ++r) {
        const int64_t s = ld_idx(ptr, pdt, r), e = ld_idx(ptr, pdt, r + 1);
        for (int64_t q = s; q < e; ++q) {
            const int64_t c = ld_idx(col, idt, q);
            if (vdt == ORC_F32) {
                const float* xr = (const float*)x + r * ldx;
                const float* yc = (const float*)y + c * ldy;
                float acc = 0.f;
                for (int64_t t = 0; t < k; ++t) acc = fmaf(xr[t], yc[t], acc);
                float v = (float)alpha * acc;
                if (data) v += ((const float*)data)[q] * (float)beta;
                ((float*)out)[q] = v;
            } else {
                const double* xr = (const double*)x + r * ldx;
                const double* yc = (const double*)y + c * ldy;
                double acc = 0.0;
                for (int64_t t = 0; t < k; ++t) acc = fma(xr[t], yc[t], acc);
                double v = alpha * acc;
                if (data) v += ((const double*)data)[q] * beta;
                ((double*)out)[q] = v;
            }
        }
    }
    return 0;
}
