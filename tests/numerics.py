"""Error measures shared by the parity tests.

The bound of every floating-point comparison is stated per row (SpMV) or per
entry (SpMM) against the FP64 oracle, scaled by the row's magnitude
sum_k |a_k * x_k| (condition-scaled relative error):

    err = |y - y_fp64| / max(sum_k |a_k x_k|, tiny)

which is what a correctly implemented floating-point dot product guarantees
whatever the cancellation inside the row.
"""

import torch

# Bounds on the condition-scaled error vs the FP64 oracle, by result dtype and
# accumulation: float32 results at most 1e-5 (wide accumulation reaches about
# one float32 rounding), float64 1e-12, half types one rounding of the type
# plus float32 accumulation.
REL_BOUND = {
    torch.float32: 1e-5,
    torch.complex64: 1e-5,
    torch.float64: 1e-12,
    torch.complex128: 1e-12,
    torch.float16: 1e-3,
    torch.bfloat16: 4e-3,
}


# Half the spacing of the subnormal numbers of each result type: rounding a
# result into the subnormal range errs by up to this much in absolute terms,
# which no relative bound covers.
SUBNORMAL_HALF_SPACING = {
    torch.float16: 2.0 ** -25,
    torch.bfloat16: 2.0 ** -134,
    torch.float32: 2.0 ** -150,
}


def scaled_error(actual, exact, mag):
    """Max over entries of |actual - exact| / max(mag, tiny) (all on CPU, float64).

    For half-precision results the subnormal rounding floor is subtracted first.
    """
    a = actual.detach().cpu()
    e = exact.detach().cpu()
    if a.numel() == 0:
        return 0.0
    if a.dtype.is_complex or e.dtype.is_complex:
        diff = (a.to(torch.complex128) - e.to(torch.complex128)).abs()
    else:
        diff = (a.to(torch.float64) - e.to(torch.float64)).abs()
        floor = SUBNORMAL_HALF_SPACING.get(a.dtype, 0.0)
        if floor:
            diff = (diff - floor).clamp(min=0.0)
    denom = mag.detach().cpu().to(torch.float64).clamp(min=1e-300)
    err = diff / denom
    # rows whose magnitude is zero must be exactly zero
    zero_rows = mag.detach().cpu() == 0
    if bool(zero_rows.any()):
        assert float(diff[zero_rows].max()) == 0.0, "row with no nonzeros is not zero"
        err = torch.where(zero_rows, torch.zeros_like(err), err)
    return float(err.max())


def ulp_distance_f32(a, b):
    """Max distance in float32 units in the last place between two float32 tensors."""
    ai = a.detach().cpu().contiguous().view(torch.int32).to(torch.int64)
    bi = b.detach().cpu().contiguous().view(torch.int32).to(torch.int64)
    # map to a monotone integer line
    ai = torch.where(ai < 0, -(ai & 0x7FFFFFFF), ai)
    bi = torch.where(bi < 0, -(bi & 0x7FFFFFFF), bi)
    return int((ai - bi).abs().max()) if ai.numel() else 0
