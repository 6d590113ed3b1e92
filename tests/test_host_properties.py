"""Property tests of the simulator's host-side tables against the oracle.

The state-machine numbering (gpu_batch_simulator.py:262-299), the flattened reaction pairs
with their n_needed rule (:186-205) and the trajectory shards are plain host logic; here they
are compared with the oracle's restatement on generated inputs.
"""

from types import SimpleNamespace

import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

from oracle.stepper import n_needed_of, sm_tables
from pystarc_b200.shard import shard_range
from pystarc_b200.simulator import flatten_pairs, state_machine

LABELS = st.one_of(st.none(), st.sampled_from(["A", "B", "C", "D", "E"]))


def _pair(i):
    return SimpleNamespace(mol1_atom_index=i, mol2_atom_index=i + 1, distance_cutoff=1.0 + i)


def _pathway(befores, afters, first, n_pairs=None, n_needed=1):
    rxns = []
    for k, (b, a) in enumerate(zip(befores, afters)):
        pairs = [_pair(k)] if n_pairs is None else [_pair(k * 10 + j) for j in range(n_pairs[k])]
        rxns.append(SimpleNamespace(name=f"r{k}", state_before=b, state_after=a,
                                    criteria=SimpleNamespace(pairs=pairs, n_needed=n_needed)))
    return SimpleNamespace(reactions=rxns, first_state=first)


@settings(max_examples=200, deadline=None)
@given(st.lists(st.tuples(LABELS, LABELS), min_size=1, max_size=8), LABELS)
def test_state_numbering_matches_oracle(pairs, first):
    befores = [b for b, _ in pairs]
    afters = [a for _, a in pairs]
    sm = state_machine(_pathway(befores, afters, first))
    if all(b is None for b in befores):
        assert sm is None  # no state_before label: the flattened-pairs mode
        return
    b, a, term = sm_tables(befores, afters, first)
    assert sm["before"] == list(b) and sm["after"] == list(a)
    assert sm["terminal"] == list(term)
    assert len(sm["states"]) == len(term)


@settings(max_examples=200, deadline=None)
@given(st.lists(st.integers(0, 4), min_size=1, max_size=6), st.integers(-1, 12))
def test_flattened_pairs_and_n_needed_match_oracle(n_pairs, n_needed):
    pw = _pathway([None] * len(n_pairs), [None] * len(n_pairs), None, n_pairs=n_pairs, n_needed=n_needed)
    rec, lig, cut, nn = flatten_pairs(pw)
    assert len(rec) == len(lig) == len(cut) == sum(n_pairs)
    assert nn == n_needed_of(n_needed, sum(n_pairs))
    # every pair of every reaction, in reaction order
    want = [k * 10 + j for k, n in enumerate(n_pairs) for j in range(n)]
    assert rec == want and lig == [w + 1 for w in want]
    np.testing.assert_array_equal(cut, [1.0 + w for w in want])


@settings(max_examples=300, deadline=None)
@given(st.integers(0, 10 ** 7), st.integers(1, 64))
def test_shards_are_contiguous_and_balanced(n_total, world):
    spans = [shard_range(n_total, r, world) for r in range(world)]
    assert spans[0][0] == 0
    for (o0, n0), (o1, _) in zip(spans, spans[1:]):
        assert o1 == o0 + n0
    assert spans[-1][0] + spans[-1][1] == n_total
    sizes = [n for _, n in spans]
    assert max(sizes) - min(sizes) <= 1
