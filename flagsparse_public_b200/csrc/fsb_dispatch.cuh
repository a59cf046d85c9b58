// fsb_dispatch.cuh -- maps the C-ABI type codes onto template instantiations.
#pragma once
#include "fsb_common.cuh"

namespace fsb {

template <class T> struct tag { using type = T; };

// (value, accumulator, output) triples that are compiled in.  Returns
// FSB_ERR_UNSUPPORTED for any other combination.
//   acc_mode NATIVE : f16/bf16->f32, f32->f32, f64->f64, c64->c64, c128->c128
//   acc_mode WIDE   : f16/bf16->f32, f32->f64, f64->f64, c64->c128, c128->c128
//   acc_mode COMP   : f16/bf16/f32 -> compensated f32
//   complex32 (c32) : float32 pairs in NATIVE and WIDE (as FlagSparse)
// Output is the value type, or f32 for f16/bf16/f32 values (precision form).
template <class F>
int dispatch_vao(int vdt, int acc_mode, int odt, F&& f) {
    const bool out_same = (odt == vdt);
    const bool out_f32 = (odt == FSB_F32);
    switch (vdt) {
    case FSB_F16:
        if (acc_mode == FSB_ACC_COMP) {
            if (out_f32) return f(tag<__half>{}, tag<comp_t>{}, tag<float>{});
            if (out_same) return f(tag<__half>{}, tag<comp_t>{}, tag<__half>{});
            break;
        }
        if (out_same) return f(tag<__half>{}, tag<float>{}, tag<__half>{});
        if (out_f32) return f(tag<__half>{}, tag<float>{}, tag<float>{});
        break;
    case FSB_BF16:
        if (acc_mode == FSB_ACC_COMP) {
            if (out_f32) return f(tag<__nv_bfloat16>{}, tag<comp_t>{}, tag<float>{});
            if (out_same) return f(tag<__nv_bfloat16>{}, tag<comp_t>{}, tag<__nv_bfloat16>{});
            break;
        }
        if (out_same) return f(tag<__nv_bfloat16>{}, tag<float>{}, tag<__nv_bfloat16>{});
        if (out_f32) return f(tag<__nv_bfloat16>{}, tag<float>{}, tag<float>{});
        break;
    case FSB_F32:
        if (!out_same) break;
        if (acc_mode == FSB_ACC_COMP) return f(tag<float>{}, tag<comp_t>{}, tag<float>{});
        if (acc_mode == FSB_ACC_WIDE) return f(tag<float>{}, tag<double>{}, tag<float>{});
        return f(tag<float>{}, tag<float>{}, tag<float>{});
    case FSB_F64:
        if (!out_same || acc_mode == FSB_ACC_COMP) break;
        return f(tag<double>{}, tag<double>{}, tag<double>{});
    case FSB_C64:
        if (!out_same || acc_mode == FSB_ACC_COMP) break;
        if (acc_mode == FSB_ACC_WIDE) return f(tag<c64_t>{}, tag<c128_t>{}, tag<c64_t>{});
        return f(tag<c64_t>{}, tag<c64_t>{}, tag<c64_t>{});
    case FSB_C128:
        if (!out_same || acc_mode == FSB_ACC_COMP) break;
        return f(tag<c128_t>{}, tag<c128_t>{}, tag<c128_t>{});
    case FSB_C32:
        if (!out_same || acc_mode == FSB_ACC_COMP) break;
        return f(tag<c32_t>{}, tag<c64_t>{}, tag<c32_t>{});
    default:
        break;
    }
    fsb_host::set_error("unsupported value/accumulate/output combination (%d, %d, %d)", vdt, acc_mode, odt);
    return FSB_ERR_UNSUPPORTED;
}

template <class F>
int dispatch_idx(int dt, F&& f) {
    if (dt == FSB_I32) return f(tag<int32_t>{});
    if (dt == FSB_I64) return f(tag<int64_t>{});
    fsb_host::set_error("index dtype code %d is not int32/int64", dt);
    return FSB_ERR_UNSUPPORTED;
}

inline int elem_size(int dt) {
    switch (dt) {
    case FSB_F16: case FSB_BF16: return 2;
    case FSB_F32: case FSB_I32: case FSB_C32: return 4;
    case FSB_F64: case FSB_C64: case FSB_I64: return 8;
    case FSB_C128: return 16;
    default: return 0;
    }
}

// Bytes of one accumulator element for (value dtype, acc mode).
inline int acc_size(int vdt, int acc_mode) {
    if (acc_mode == FSB_ACC_COMP) return 8;
    switch (vdt) {
    case FSB_F16: case FSB_BF16: return 4;
    case FSB_F32: return acc_mode == FSB_ACC_WIDE ? 8 : 4;
    case FSB_F64: return 8;
    case FSB_C64: return acc_mode == FSB_ACC_WIDE ? 16 : 8;
    case FSB_C128: return 16;
    case FSB_C32: return 8;
    default: return 0;
    }
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

inline int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

// Merge-path scratch layout (shared by SpMV tiles and SpMM units):
//   int64 carry_row[n_units] | A carry_val[n_units * width] | A head_val[n_units * width]
struct MergeScratch {
    int64_t* carry_row;
    void* carry_val;
    void* head_val;
};
inline int64_t merge_scratch_bytes(int64_t n_units, int64_t width, int acc_bytes) {
    int64_t b = align_up(n_units * 8, 256);
    b += align_up(n_units * width * acc_bytes, 256);
    b += align_up(n_units * width * acc_bytes, 256);
    return b;
}
inline MergeScratch merge_scratch_carve(void* ws, int64_t n_units, int64_t width, int acc_bytes) {
    char* p = static_cast<char*>(ws);
    MergeScratch s;
    s.carry_row = reinterpret_cast<int64_t*>(p);
    p += align_up(n_units * 8, 256);
    s.carry_val = p;
    p += align_up(n_units * width * acc_bytes, 256);
    s.head_val = p;
    return s;
}

}  // namespace fsb
