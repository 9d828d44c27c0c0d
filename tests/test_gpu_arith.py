"""The two quotient modes of the stage kernel give the same bits.

GO_ARITH_RCP (the default) evaluates the reference's quotients a / b as
a * rcp.approx.ftz(b); GO_ARITH_EXACT keeps a / b as the reference compiles
it (div.full.f32 under --prec-div=false, CDKLM16.py:196-200).  The library's
go_check_quotients returns both, compiled with the stage kernel's flags.
Denominators are the ones the scheme divides by in those quotients (depths
h >= desing_eps, 1 + C and 1 + C/2, ap - am >= flux_slope_eps, 2g, dx, dy),
with numerators over the whole normal range, plus near-cutoff depths, the
land value 1e20 and denormal-adjacent operands.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from SWESimulators import _native  # noqa: E402


def quotients(a, b):
    lib = _native.load()
    ta = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    tb = torch.from_numpy(np.ascontiguousarray(b, np.float32)).cuda()
    qd = torch.empty_like(ta)
    qr = torch.empty_like(ta)
    s = torch.cuda.current_stream()
    _native.check(lib.go_check_quotients(ctypes.c_void_p(s.cuda_stream), _native.ptr(ta), _native.ptr(tb),
                                         int(ta.numel()), _native.ptr(qd), _native.ptr(qr)))
    torch.cuda.synchronize()
    return qd.cpu().numpy(), qr.cpu().numpy()


def log_uniform(rng, lo, hi, n, signed=False):
    x = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    if signed:
        x *= rng.choice([-1.0, 1.0], n)
    return x.astype(np.float32)


def mismatches(a, b):
    qd, qr = quotients(a, b)
    bad = (qd.view(np.uint32) != qr.view(np.uint32)) & ~(np.isnan(qd) & np.isnan(qr))
    return int(bad.sum()), qd, qr, bad


def test_scheme_denominators_bit_identical():
    rng = np.random.default_rng(7)
    n = 1 << 22
    nums = log_uniform(rng, 1e-37, 1e37, n, signed=True)
    dens = np.concatenate([
        log_uniform(rng, 0.1, 1.0e4, n // 4),               # depths h >= desing_eps (0.1)
        (1.0 + log_uniform(rng, 1e-9, 10.0, n // 8)),        # 1 + C
        (1.0 + 0.5 * log_uniform(rng, 1e-9, 10.0, n // 8)),  # 1 + C/2
        log_uniform(rng, 0.1, 1.0e3, n // 4),                # ap - am >= flux_slope_eps (0.1)
        np.full(n // 8, np.float32(2.0) * np.float32(9.81)),  # 2g
        np.full(n // 16, 500.0), np.full(n // 16, 200.0),  # dx, dy
    ]).astype(np.float32)[:n]
    nbad, qd, qr, bad = mismatches(nums, dens)
    assert nbad == 0, (nums[bad][:5], dens[bad][:5], qd[bad][:5], qr[bad][:5])
    # every bit pattern of the mantissa for one numerator and one denominator decade
    m = np.arange(1 << 23, dtype=np.uint32)
    den = ((np.uint32(127) << 23) | m).view(np.float32)        # [1, 2)
    num = np.full_like(den, np.float32(3.0))
    assert mismatches(num, den)[0] == 0
    assert mismatches(den, np.full_like(den, np.float32(19.62)))[0] == 0


def test_edge_operands():
    rng = np.random.default_rng(8)
    n = 1 << 20
    cases = {
        # depths near the dry cut-off (1e-5) and the desingularisation depth
        "near_cutoff": (log_uniform(rng, 1e-6, 1e3, n, signed=True), log_uniform(rng, 1e-5, 0.2, n)),
        # the land value as a numerator (eta of a land cell is the dry flag)
        "land": (np.full(n, 1.0e20, np.float32) * rng.choice([-1, 1], n).astype(np.float32),
                 log_uniform(rng, 0.1, 1e4, n)),
        # results at the edge of the normal range (flushed to zero below it)
        "tiny_results": (log_uniform(rng, 1e-38, 1e-35, n, signed=True), log_uniform(rng, 0.1, 1e4, n)),
        "denormal_adjacent_num": (log_uniform(rng, 1.1754944e-38, 1e-37, n, signed=True),
                                  log_uniform(rng, 0.5, 2.0, n)),
    }
    report = {}
    for name, (a, b) in cases.items():
        report[name] = mismatches(a, b)[0]
    print("quotient mode mismatches per case:", report)
    assert all(v == 0 for v in report.values()), report
