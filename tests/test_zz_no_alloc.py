"""llg_run_noalloc, the entry point for callers that cannot allocate device memory: its output must
equal the allocating entry point's (bit-exact residues) on two calls in a row, the second one
starting from whatever the first left in the shared fixed-size device array. Kept in a file that
pytest collects last, so that a failure here comes after every other test has run."""
import pytest

pytestmark = pytest.mark.gpu


def _residue_via_noalloc(gpu, torch, p, k, n):
    out = torch.full((n,), -7, dtype=torch.int32, device="cuda")  # caller-owned output buffer
    stream = torch.cuda.current_stream().cuda_stream
    err = gpu.run_noalloc(p, k, n, out.data_ptr(), stream)
    torch.cuda.synchronize()
    return gpu.residue_from_digits(p, n, out.cpu().tolist()), err


def test_noalloc_matches_allocating_entry_point(gpu):
    torch = pytest.importorskip("torch")
    # N = 65536 (rows of 2^8), 32768 (rows of 2^7), 16384 (rows of 2^6): each split of the array
    cases = [(1257787, 1000, 65536), (600011, 300, 32768), (300007, 257, 16384), (300007, 100, 16384)]
    for p, k, n in cases:  # calls in a row, different sizes, then a repeat: no state may leak between them
        want = gpu.run(p, iters=k, n=n, want_words=True)
        (z, r64, words), err = _residue_via_noalloc(gpu, torch, p, k, n)
        assert words == want["words"] and r64 == want["res64"], (p, k, n)
        assert err <= 0.4


def test_noalloc_rejects_lengths_beyond_its_array(gpu):
    torch = pytest.importorskip("torch")
    out = torch.zeros(1 << 17, dtype=torch.int32, device="cuda")
    with pytest.raises(gpu.LlgError) as e:
        gpu.run_noalloc(2000003, 10, 1 << 17, out.data_ptr())
    assert e.value.code == 4  # LLG_E_UNSUPPORTED
