"""Device integer prepare steps: the stable radix sort (fsb_stable_sort) and
run starts (fsb_run_starts) against torch.sort(stable=True) and the nonzero
expression they replace -- integer results, compared bit for bit."""

import pytest
import torch

from flagsparse_public_b200 import _native as nat
from flagsparse_public_b200 import _plan

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _check_sort(keys, key_bound=None):
    got_k, got_o = _plan.stable_sort(keys, key_bound=key_bound)
    ref_k, ref_o = torch.sort(keys, stable=True)
    assert torch.equal(got_k, ref_k)
    assert torch.equal(got_o, ref_o)


@pytest.mark.parametrize("n", [1, 2, 255, 4095, 4096, 4097, 100003, 1 << 20])
@pytest.mark.parametrize("bound", [1, 2, 3, 256, 257, 70000, 2 ** 31 - 1])
def test_sort_int32_bounded(n, bound):
    g = torch.Generator(device=DEV).manual_seed(n * 7 + bound)
    keys = torch.randint(0, bound, (n,), generator=g, device=DEV, dtype=torch.int32)
    _check_sort(keys, key_bound=bound)


@pytest.mark.parametrize("n", [1, 5000, 300001])
def test_sort_int64_lexicographic_keys(n):
    g = torch.Generator(device=DEV).manual_seed(n)
    n_rows, n_cols = 1 << 20, 3 * (1 << 18)
    row = torch.randint(0, n_rows, (n,), generator=g, device=DEV)
    col = torch.randint(0, n_cols, (n,), generator=g, device=DEV)
    row[: n // 3] = row[0]  # many equal rows and duplicate keys
    col[: n // 5] = col[0]
    _check_sort(row * n_cols + col, key_bound=n_rows * n_cols)


@pytest.mark.parametrize("dtype", [torch.int32, torch.int64])
def test_sort_full_width_signed(dtype):
    info = torch.iinfo(dtype)
    g = torch.Generator(device=DEV).manual_seed(11)
    keys = torch.randint(info.min, info.max, (77777,), generator=g, device=DEV, dtype=dtype)
    keys[:10] = torch.tensor([info.min, info.max, 0, -1, 1, info.min, info.max, -1, 0, 5], dtype=dtype)
    _check_sort(keys)
    _check_sort(keys % 100)  # negative and positive small keys, full width


@pytest.mark.parametrize("pattern", ["equal", "sorted", "reversed"])
def test_sort_ordered_inputs(pattern):
    n = 50000
    keys = {"equal": torch.full((n,), 42, dtype=torch.int64),
            "sorted": torch.arange(n, dtype=torch.int64) // 3,
            "reversed": torch.arange(n, 0, -1, dtype=torch.int64) // 7}[pattern].to(DEV)
    _check_sort(keys, key_bound=n + 1)
    _check_sort(keys)


def test_sort_empty_and_workspace_errors():
    k, o = _plan.stable_sort(torch.empty(0, dtype=torch.int32, device=DEV), key_bound=10)
    assert k.numel() == 0 and o.numel() == 0 and o.dtype == torch.int64
    lib = nat.library()
    assert lib.fsb_sort_workspace_bytes(10, nat.FSB_I32, 33) == -1
    assert lib.fsb_sort_workspace_bytes(10, nat.FSB_F32, 8) == -1
    keys = torch.arange(10, dtype=torch.int32, device=DEV)
    order = torch.empty(10, dtype=torch.int64, device=DEV)
    rc = lib.fsb_stable_sort(nat.ptr(keys), nat.FSB_I32, 10, 8, None, nat.ptr(order), None, 0,
                             nat.stream_handle(keys.device))
    assert rc == nat.FSB_ERR_WORKSPACE


def _runs_ref(keys, dtype):
    n = keys.numel()
    breaks = torch.nonzero(keys[1:] != keys[:-1], as_tuple=False).flatten().to(dtype) + 1
    return torch.cat([torch.zeros(1, dtype=dtype, device=keys.device), breaks,
                      torch.tensor([n], dtype=dtype, device=keys.device)])


@pytest.mark.parametrize("n", [1, 2, 4096, 4097, 123457])
@pytest.mark.parametrize("key_dtype", [torch.int32, torch.int64])
@pytest.mark.parametrize("out_dtype", [torch.int32, torch.int64])
def test_run_starts(n, key_dtype, out_dtype):
    g = torch.Generator(device=DEV).manual_seed(n)
    keys, _ = torch.sort(torch.randint(0, max(1, n // 5), (n,), generator=g, device=DEV).to(key_dtype))
    got = _plan.run_starts(keys, out_dtype)
    assert got.dtype == out_dtype and torch.equal(got, _runs_ref(keys, out_dtype))
    for special in (torch.zeros(n, dtype=key_dtype, device=DEV), torch.arange(n, dtype=key_dtype, device=DEV)):
        assert torch.equal(_plan.run_starts(special, out_dtype), _runs_ref(special, out_dtype))
    assert _plan.run_starts(keys[:0], out_dtype) is None
