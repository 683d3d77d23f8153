"""sbx_csr_build_noalloc (static device scratch) against sbx_csr_build, through the C ABI.

Collected last on purpose (file name): it must pass on a device where every other test
has already run, as well as alone.
"""
import numpy as np
import pytest

from softbox_b200.runtime import Context, LIB

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SBX_EINVAL = -1
MAX_ITEMS = 1 << 20
MAX_ROWS = 1 << 22


def _keys(seed, n, rows):
    rng = np.random.default_rng(seed)
    k = rng.integers(0, rows, n, dtype=np.int32)
    k[rng.random(n) < 0.2] = -1          # unbound items are skipped, as in the reference
    return k


def _build(ctx, name, keys, rows):
    n = keys.size
    d_keys = torch.from_numpy(keys).cuda()
    cnt = torch.full((rows,), 7, dtype=torch.int32, device="cuda")     # garbage: the call clears it
    off = torch.full((rows + 1,), -5, dtype=torch.int32, device="cuda")
    lst = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx(name, d_keys.data_ptr(), n, rows, cnt.data_ptr(), off.data_ptr(), lst.data_ptr())
    ctx.sync()
    return cnt.cpu().numpy(), off.cpu().numpy(), lst.cpu().numpy()


@pytest.mark.parametrize("n,rows", [(6400, 20000), (200_000, 4096), (MAX_ITEMS, 1 << 16), (MAX_ITEMS, MAX_ROWS)])
def test_noalloc_matches_csr_build_twice(n, rows):
    ref_ctx, ctx = Context(0), Context(0)
    try:
        for seed in (1, 2):   # two calls in a row: the second must not see the first's scratch
            keys = _keys(seed * 7919 + n, n, rows)
            want = _build(ref_ctx, "sbx_csr_build", keys, rows)
            got = _build(ctx, "sbx_csr_build_noalloc", keys, rows)
            for w, g, what in zip(want, got, ("rowCount", "rowOffsets", "rowList")):
                assert np.array_equal(w, g), f"{what} differs (seed {seed})"
            assert got[1][-1] == int((keys >= 0).sum())
    finally:
        ref_ctx.close()
        ctx.close()


def test_noalloc_takes_no_device_memory():
    ctx = Context(0)
    try:
        keys = _keys(5, 50_000, 10_000)
        _build(ctx, "sbx_csr_build_noalloc", keys, 10_000)     # first call on the device: set-up
        d_keys = torch.from_numpy(keys).cuda()
        cnt = torch.zeros(10_000, dtype=torch.int32, device="cuda")
        off = torch.zeros(10_001, dtype=torch.int32, device="cuda")
        lst = torch.zeros(keys.size, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        scratch0 = ctx.scratch_bytes()
        free0, _ = torch.cuda.mem_get_info()
        for _ in range(3):
            ctx("sbx_csr_build_noalloc", d_keys.data_ptr(), keys.size, 10_000, cnt.data_ptr(), off.data_ptr(),
                lst.data_ptr())
        ctx.sync()
        free1, _ = torch.cuda.mem_get_info()
        # the context's own scratch did not grow (the direct check) ...
        assert ctx.scratch_bytes() == scratch0
        # ... and the device's free memory did not move (a secondary check: another process
        # on the same GPU could move it)
        assert free1 == free0
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_the_static_scratch():
    ctx = Context(0)
    try:
        buf = torch.zeros(16, dtype=torch.int32, device="cuda")
        p = buf.data_ptr()
        assert ctx.raw("sbx_csr_build_noalloc", p, MAX_ITEMS + 1, 8, p, p, p) == SBX_EINVAL
        assert "exceeds the static scratch limit" in ctx.last_error()
        assert ctx.raw("sbx_csr_build_noalloc", p, 4, MAX_ROWS + 1, p, p, p) == SBX_EINVAL
        assert "exceeds the static scratch limit" in ctx.last_error()
        # the context stays usable after a rejection
        keys = _keys(9, 1000, 64)
        want = _build(ctx, "sbx_csr_build", keys, 64)
        got = _build(ctx, "sbx_csr_build_noalloc", keys, 64)
        for w, g in zip(want, got):
            assert np.array_equal(w, g)
    finally:
        ctx.close()


def test_noalloc_out_of_range_key_is_skipped_and_reported():
    """A key at or past the row count indexes no row: the item is skipped (the static
    scratch is not written past its rows), the next sync reports SBX_EINVAL, and the
    outputs equal the build of the same keys with that item unbound."""
    ctx = Context(0)
    try:
        rows = 4096
        keys = _keys(11, 100_000, rows)
        bad = keys.copy()
        bad[777] = rows          # one past the last row
        bad[5000] = rows + 12345
        d_keys = torch.from_numpy(bad).cuda()
        cnt = torch.zeros(rows, dtype=torch.int32, device="cuda")
        off = torch.zeros(rows + 1, dtype=torch.int32, device="cuda")
        lst = torch.full((bad.size,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        assert ctx.raw("sbx_csr_build_noalloc", d_keys.data_ptr(), bad.size, rows, cnt.data_ptr(), off.data_ptr(),
                       lst.data_ptr()) == 0
        assert ctx.raw("sbx_ctx_sync") == SBX_EINVAL
        assert "row count" in ctx.last_error()
        assert ctx.raw("sbx_ctx_sync") == 0          # reported once
        fixed = bad.copy()
        fixed[bad >= rows] = -1
        want = _build(ctx, "sbx_csr_build", fixed, rows)
        assert np.array_equal(want[0], cnt.cpu().numpy())
        assert np.array_equal(want[1], off.cpu().numpy())
        n_valid = int(want[1][-1])
        assert np.array_equal(want[2][:n_valid], lst.cpu().numpy()[:n_valid])
    finally:
        ctx.close()
