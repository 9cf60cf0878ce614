"""dsb_boxcar_argmax_noalloc: the boxcar S/N argmax for callers that cannot
allocate device memory.

Such a caller (a host that gives all of the GPU's memory to its own fixed
arena, or a real-time loop where an allocation or free would stall every
stream on the device) cannot hand dsb_multi_boxcar_argmax the prefix-sum
buffer it reads.  The no-alloc entry point keeps that buffer in a fixed
array inside the library instead.  These tests call it through the C ABI
twice in a row, the second time on a smaller problem so that the first
call's prefix sums are still in the array, and check each result against
the allocating pair dsb_padded_cumsum + dsb_multi_boxcar_argmax on the same
inputs.  The file sorts last so that it also runs after every other test
has used the library on the same device.
"""

import numpy as np
import pytest
import torch

from dsb200 import _lib

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 16 << 20


def _case(n, inner, max_w, n_out, t_base, f16, seed, dev):
    g = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.randn((n, inner), generator=g, dtype=torch.float32)
    x = x.to(torch.float16 if f16 else torch.float32).to(dev)
    widths = [1 << i for i in range(max_w.bit_length()) if (1 << i) <= max_w]
    offs = [max_w // 2 - w // 2 for w in widths]
    sinv = [1.0 / np.sqrt(w) for w in widths]
    w_d = torch.tensor(widths, dtype=torch.int32, device=dev)
    o_d = torch.tensor(offs, dtype=torch.int32, device=dev)
    s_d = torch.tensor(sinv, dtype=torch.float32, device=dev)
    return x, w_d, o_d, s_d


def _run_pair(L, x, f16, n, inner, max_w, w_d, o_d, s_d, n_out, t_base, out_f16, stream):
    dev = x.device
    cs = torch.empty((n + max_w, inner), dtype=torch.float32, device=dev)
    _lib.check(L.dsb_padded_cumsum(_lib.ptr(x), int(f16), n, inner, max_w, _lib.ptr(cs), stream),
               "dsb_padded_cumsum")
    mx = torch.empty((n_out, inner), dtype=torch.float16 if out_f16 else torch.float32, device=dev)
    win = torch.empty((n_out, inner), dtype=torch.int16, device=dev)
    _lib.check(L.dsb_multi_boxcar_argmax(_lib.ptr(cs), inner, _lib.ptr(w_d), _lib.ptr(o_d),
                                         _lib.ptr(s_d), w_d.numel(), n_out, t_base, _lib.ptr(mx),
                                         int(out_f16), _lib.ptr(win), stream),
               "dsb_multi_boxcar_argmax")
    return mx, win


def _run_noalloc(L, x, f16, n, inner, max_w, w_d, o_d, s_d, n_out, t_base, out_f16, stream):
    dev = x.device
    mx = torch.empty((n_out, inner), dtype=torch.float16 if out_f16 else torch.float32, device=dev)
    win = torch.empty((n_out, inner), dtype=torch.int16, device=dev)
    _lib.check(L.dsb_boxcar_argmax_noalloc(_lib.ptr(x), int(f16), n, inner, max_w, _lib.ptr(w_d),
                                           _lib.ptr(o_d), _lib.ptr(s_d), w_d.numel(), n_out,
                                           t_base, _lib.ptr(mx), int(out_f16), _lib.ptr(win),
                                           stream),
               "dsb_boxcar_argmax_noalloc")
    return mx, win


def test_noalloc_matches_allocating_pair_on_two_calls():
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = _lib.lib()
    stream = _lib.stream_of(dev)
    # (n, inner, max_w, n_out, t_base, f16 in, f16 out): the first call fills
    # most of the array, the second is smaller and reads over its leftovers.
    cases = [(256, 12000, 16, 240, 8, False, False, 11),
             (96, 5000, 8, 80, 16, True, True, 12)]
    for (n, inner, max_w, n_out, t_base, f16, out_f16, seed) in cases:
        assert (n + max_w) * inner * 4 <= SCRATCH_BYTES
        x, w_d, o_d, s_d = _case(n, inner, max_w, n_out, t_base, f16, seed, dev)
        got_mx, got_win = _run_noalloc(L, x, f16, n, inner, max_w, w_d, o_d, s_d, n_out, t_base,
                                       out_f16, stream)
        ref_mx, ref_win = _run_pair(L, x, f16, n, inner, max_w, w_d, o_d, s_d, n_out, t_base,
                                    out_f16, stream)
        torch.cuda.synchronize(dev)
        # the same two kernels on the same inputs: the same bits
        assert torch.equal(got_mx, ref_mx)
        assert torch.equal(got_win, ref_win)


def test_noalloc_rejects_sizes_beyond_its_array():
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = _lib.lib()
    n, max_w = 64, 16
    inner = SCRATCH_BYTES // 4 // (n + max_w) + 1          # one column too many
    x = torch.zeros(1, dtype=torch.float32, device=dev)    # never read: rejected first
    w_d = torch.ones(1, dtype=torch.int32, device=dev)
    o_d = torch.full((1,), max_w // 2, dtype=torch.int32, device=dev)
    s_d = torch.ones(1, dtype=torch.float32, device=dev)
    out = torch.zeros(1, dtype=torch.float32, device=dev)
    win = torch.zeros(1, dtype=torch.int16, device=dev)
    rc = L.dsb_boxcar_argmax_noalloc(_lib.ptr(x), 0, n, inner, max_w, _lib.ptr(w_d), _lib.ptr(o_d),
                                     _lib.ptr(s_d), 1, n, 0, _lib.ptr(out), 0, _lib.ptr(win),
                                     _lib.stream_of(dev))
    assert rc == 5                                          # DSB_E_CAPACITY
    assert b"capacity" in L.dsb_strerror(rc)


def test_noalloc_rejects_a_size_whose_row_count_overflows_32_bits():
    """n + max_w above 2^31 (n = 2^30 + 1, max_w = 2^30) with one column: the
    row count is formed in 64 bits and rejected before any launch, so the
    placeholder buffers are never touched."""
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = _lib.lib()
    n, max_w = (1 << 30) + 1, 1 << 30
    x = torch.zeros(1, dtype=torch.float32, device=dev)
    w_d = torch.ones(1, dtype=torch.int32, device=dev)
    o_d = torch.zeros(1, dtype=torch.int32, device=dev)
    s_d = torch.ones(1, dtype=torch.float32, device=dev)
    out = torch.zeros(1, dtype=torch.float32, device=dev)
    win = torch.zeros(1, dtype=torch.int16, device=dev)
    rc = L.dsb_boxcar_argmax_noalloc(_lib.ptr(x), 0, n, 1, max_w, _lib.ptr(w_d), _lib.ptr(o_d),
                                     _lib.ptr(s_d), 1, 1, 0, _lib.ptr(out), 0, _lib.ptr(win),
                                     _lib.stream_of(dev))
    assert rc == 5                                          # DSB_E_CAPACITY


def test_noalloc_flags_widths_reading_outside_its_rows():
    """A width past max_w would read prefix rows beyond this call's n + max_w
    (leftovers of an earlier, larger call in the shared array): those outputs
    come back NaN with winner -1; outputs whose rows are in range are exact."""
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = _lib.lib()
    stream = _lib.stream_of(dev)
    n, inner, max_w, n_out, t_base = 64, 1000, 8, 64, 0
    x, w_d, o_d, s_d = _case(n, inner, max_w, n_out, t_base, False, 5, dev)
    bad_w = w_d.clone()
    bad_w[-1] = 4 * max_w                                  # past the padding at the end
    mx, win = _run_noalloc(L, x, False, n, inner, max_w, bad_w, o_d, s_d, n_out, t_base, False,
                           stream)
    torch.cuda.synchronize(dev)
    off_last = int(o_d[-1].item())
    rows = n + max_w
    bad_t = [t for t in range(n_out) if t + t_base + off_last + 4 * max_w >= rows]
    good_t = [t for t in range(n_out) if t not in bad_t]
    assert bad_t and good_t
    assert torch.isnan(mx[bad_t]).all() and (win[bad_t] == -1).all()
    # the reference: the allocating pair over a prefix buffer with room for
    # every row the widened kernel reads (the rows past n + max_w are NaN)
    cs = torch.full((n + 5 * max_w, inner), float("nan"), dtype=torch.float32, device=dev)
    _lib.check(L.dsb_padded_cumsum(_lib.ptr(x), 0, n, inner, max_w, _lib.ptr(cs), stream),
               "dsb_padded_cumsum")
    ref_mx = torch.empty((n_out, inner), dtype=torch.float32, device=dev)
    ref_win = torch.empty((n_out, inner), dtype=torch.int16, device=dev)
    assert n_out - 1 + t_base + off_last + 4 * max_w < cs.shape[0]
    _lib.check(L.dsb_multi_boxcar_argmax(_lib.ptr(cs), inner, _lib.ptr(bad_w), _lib.ptr(o_d),
                                         _lib.ptr(s_d), bad_w.numel(), n_out, t_base,
                                         _lib.ptr(ref_mx), 0, _lib.ptr(ref_win), stream),
               "dsb_multi_boxcar_argmax")
    torch.cuda.synchronize(dev)
    assert torch.equal(mx[good_t], ref_mx[good_t]) and torch.equal(win[good_t], ref_win[good_t])
