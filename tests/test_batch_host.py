"""Host-side checks of the batched slab engine (no GPU): the host Philox (rng.py) against
the oracle's, the uneven 256-instance batch's parameter ranges and determinism, the bank slot
plan, and the ledger field numbering against include/imcb200.h."""
import pathlib
import re

import numpy as np

from oracle import oracle as O
from radtranbook_b200 import _lib, batch, rng as host_rng

ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_host_philox_matches_oracle():
    rng = np.random.default_rng(3)
    ctr = rng.integers(0, 2 ** 32, size=(64, 4), dtype=np.uint64).astype(np.uint32)
    key = (0x1234567, 0x89ABCDEF)
    got = host_rng.philox4x32_10(ctr, key[0] | (key[1] << 32))
    for q in range(len(ctr)):
        np.testing.assert_array_equal(got[q], O.philox(ctr[q], key))


def test_uneven_batch_parameters():
    s = batch.uneven_slab_batch()
    assert s.K == 256
    assert s.n_cells.min() >= 50 and s.n_cells.max() <= 800
    assert 0.05 <= s.length.min() and s.length.max() <= 1.0
    N = s.n_target + s.n_boundary
    assert N.min() >= 10 ** 4 - 1 and N.max() <= 10 ** 6
    assert np.all(s.n_max == 4 * N)
    assert 10.0 <= s.opacity_a.min() and s.opacity_a.max() <= 1000.0
    assert np.all(s.opacity_p == -3.0)
    assert 0.05 <= s.cv.min() and s.cv.max() <= 1.0
    assert 0.3 <= s.face_T[:, 0].min() and s.face_T[:, 0].max() <= 2.0
    assert np.all(s.face_T[:, 1] == 0.0) and np.all(s.reflect == 0)
    # log-uniform particle counts: about half the instances below 10^5
    assert 0.3 < np.mean(N < 1e5) < 0.7
    # one master seed decides everything; distinct keys per instance
    s2 = batch.uneven_slab_batch()
    np.testing.assert_array_equal(s.seed, s2.seed)
    np.testing.assert_array_equal(s.n_cells, s2.n_cells)
    assert len(set(int(x) for x in s.seed)) == 256
    assert not np.array_equal(batch.uneven_slab_batch(master_seed=1).seed, s.seed)


def test_slot_plan_holds_census_and_sources():
    s = batch.uneven_slab_batch(n_inst=32, particle_scale=0.01)
    off, new_max, total_new = batch.slot_plan(s)
    slots = np.diff(off)
    census_cap = slots - new_max
    assert np.all(census_cap >= s.n_max + s.n_cells)
    assert np.all(census_cap >= s.n_target + s.n_cells)  # the initial census fits
    assert total_new == new_max.sum()
    assert np.all(new_max == s.n_boundary + s.n_target + s.n_cells)  # one source face


def test_ledger_fields_match_header():
    txt = (ROOT / "include" / "imcb200.h").read_text()
    fields = dict((m.group(1), int(m.group(2))) for m in re.finditer(r"IMC_BL_(\w+)\s*=\s*(\d+)", txt))
    for name, value in fields.items():
        assert getattr(_lib, "BL_" + name) == value, name
    assert fields["N"] == _lib.BL_N
