"""The synthetic workload generators match the shapes they stand in for."""
import numpy as np

from hspz_b200 import synth


def test_repeat_dense_composition():
    rng = np.random.default_rng(1)
    fam = synth.repeat_families(rng, n_fam=50)
    assert all(300 <= f.size <= 6000 for f in fam)
    g = synth.repeat_genome(rng, 2_000_000, fam)
    assert g.size == 2_000_000 and set(np.unique(g).tolist()) <= set(b"ACGT")
    # copies of the families and tandem arrays make seed words recur: the
    # mean bucket size a 12-mer lands in is far above an i.i.d. genome's
    def collision_mass(s):
        codes = np.searchsorted(np.frombuffer(b"ACGT", np.uint8), s).astype(np.int64)
        k = np.zeros(s.size - 11, dtype=np.int64)
        for i in range(12):
            k = (k << 2) | codes[i: i + k.size]
        c = np.bincount(k, minlength=1 << 24).astype(np.float64)
        return (c * c).sum() / k.size
    bg = synth.random_genome(np.random.default_rng(2), 2_000_000)
    assert collision_mass(g) > 2.0 * collision_mass(bg)


def test_config4_small_scale():
    t, q = synth.config4(scale=0.002)
    assert t.size == q.size == 2_000_000
    lower = (t >= 97).mean()
    assert 0.05 < lower < 0.2  # ~10% soft-masked


def test_serving_request_lengths_and_planted_homology():
    rng = np.random.default_rng(3)
    L = synth.request_lengths(rng, 20_000)
    assert L.max() <= 5_000_000 and L.min() >= 1000
    assert 180_000 < np.median(L) < 220_000
    target = synth.config5_target(scale=0.001)
    assert target.size == 3_000_000
    q = synth.serving_request(rng, target, 50_000)
    assert q.size == 50_000


def test_soft_mask_large_path_equals_array_path(monkeypatch):
    a = synth.random_bases(np.random.default_rng(4), 300_000)
    want = synth.soft_mask(np.random.default_rng(5), a)
    # force the loop used for genome-sized inputs
    n = a.size
    rng = np.random.default_rng(5)
    k = int(n * 0.10 / 275.0) + 1
    starts, lens = rng.integers(0, n, k), rng.integers(50, 501, k)
    got = a.copy()
    for s, l in zip(starts.tolist(), lens.tolist()):
        got[s: s + l] |= 0x20
    assert np.array_equal(got, want)
