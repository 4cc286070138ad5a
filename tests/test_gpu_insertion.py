"""Random insertion with the overlap tests on the GPU (sc_insert_filaments_gpu):
batched candidates drawn at the stream positions the sequential insertion
would give them, the first overlapping one ending each batch.  The result
is the host insertion's, bit for bit -- and so the oracle's restatement of
the reference's insertion (tests/test_oracle.py) -- on isotropic, nematic,
uneven-length, 2D and dense cases (the dense ones reject often, so batches
end early and shrink)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _both(n_dim, R, seed, nb, lengths, lp, insertion="random"):
    import simcore_b200 as sc
    host = sc.insert_filaments(n_dim, R, seed, nb, lengths, lp, insertion=insertion)
    gpu = sc.insert_filaments(n_dim, R, seed, nb, lengths, lp, insertion=insertion, device=0)
    return host, gpu


@pytest.mark.parametrize("name,scale", [("A", 1.0), ("B", 0.1), ("C", 0.02), ("E", 0.05)])
def test_gpu_insertion_is_the_host_insertion(name, scale):
    from simcore_b200 import workloads
    calls = []
    real = workloads._library_insert

    def spy(*a, **kw):
        calls.append((a, kw))
        return real(*a, **kw)

    workloads.make(name, scale, seed=7, insert=spy)
    (a, kw), = calls
    host, gpu = _both(*a, insertion=kw.get("insertion", "random"))
    assert np.array_equal(host, gpu)


def test_gpu_insertion_of_2d_systems():
    from simcore_b200 import workloads
    counts = workloads.replica_counts("D", n_replicas=3, seed=8)
    for r, n in enumerate(counts):
        side = np.sqrt(n * (16 + np.pi / 4) / 0.1)
        nb = np.full(n, 16, dtype=np.int32)
        host, gpu = _both(2, 0.5 * side, 8000 + r, nb, nb.astype(float), np.full(n, 200.0))
        assert np.array_equal(host, gpu)


@pytest.mark.parametrize("n_dim", [3, 2])
def test_gpu_insertion_dense_with_rejections(n_dim):
    """A dense box where many attempts overlap: every rejection ends a
    batch, and the result is still the sequential one."""
    n = 250 if n_dim == 3 else 240
    R = 9.0 if n_dim == 3 else 34.0
    nb = np.full(n, 6, dtype=np.int32)
    host, gpu = _both(n_dim, R, 11, nb, nb.astype(float), np.full(n, 20.0))
    assert np.array_equal(host, gpu)
