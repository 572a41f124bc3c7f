"""hpt_compact_noalloc (device buffers, static scratch, no allocation)
against hpt_compact, through the C ABI.

Collected last on purpose: it must pass both in a fresh process and after
every other GPU test has run in the same process."""
import numpy as np
import pytest

import hptracing_b200 as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda(built):
    torch = pytest.importorskip("torch")
    if H.device_count() == 0 or not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _noalloc(torch, flags, stream=None):
    """Runs hpt_compact_noalloc on device copies of flags (on `stream`, else
    torch's current stream); returns (status, count, indices)."""
    n = len(flags)
    d_flags = torch.from_numpy(flags.view(np.int32)).cuda()
    d_out = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    d_count = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    stream = stream or torch.cuda.current_stream()
    stream.wait_stream(torch.cuda.current_stream())  # inputs written on the current stream
    st = H.lib().hpt_compact_noalloc(d_flags.data_ptr(), n, d_out.data_ptr(),
                                     d_count.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    count = int(d_count.item())
    return st, count, d_out[:max(count, 0)].cpu().numpy()


def test_noalloc_matches_compact_on_consecutive_calls(torch_cuda):
    rng = np.random.default_rng(11)
    # The second call is smaller than the first: counts the first call left
    # in the shared scratch must not leak into the second.
    for n, density in ((3_000_001, 0.37), (100_003, 0.81), (0, 0.5)):
        flags = (rng.random(n) < density).astype(np.uint32)
        want = H.compact(flags)
        st, count, got = _noalloc(torch_cuda, flags)
        assert st == 0, H.lib().hpt_last_error()
        assert count == len(want)
        assert np.array_equal(got, want)


def test_noalloc_on_a_side_stream(torch_cuda):
    """The work is enqueued on the caller's stream: on a side stream, at the
    limit size and at a ragged one, the results equal hpt_compact's."""
    rng = np.random.default_rng(12)
    side = torch_cuda.cuda.Stream()
    for n, density in ((8192 * 4096, 0.5), (4097, 0.02)):
        flags = (rng.random(n) < density).astype(np.uint32)
        want = H.compact(flags)
        st, count, got = _noalloc(torch_cuda, flags, side)
        assert st == 0, H.lib().hpt_last_error()
        assert count == len(want)
        assert np.array_equal(got, want)


def test_noalloc_rejects_sizes_beyond_its_scratch(torch_cuda):
    L = H.lib()
    limit = 8192 * 4096
    d = torch_cuda.zeros(1, dtype=torch_cuda.int32, device="cuda")
    st = L.hpt_compact_noalloc(d.data_ptr(), limit + 1, d.data_ptr(), d.data_ptr(), None)
    assert st == 1
    assert b"exceeds the limit" in L.hpt_last_error()
