"""Batched commitment of columns of mixed sizes (gs_commit_plan_*) against the
oracle: every extended column bit-exact, the Merkle root equal to the
oracle's MerkleProver::commit over the extended columns, eager and graph
replays identical, and a second run with other inputs (graph replay with
rewritten input pointers) still exact."""
import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = O.P


@pytest.fixture(scope="module")
def mod():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpustark import backend
    return backend


def expected(cols, logs, blowup):
    ext = [O.evaluate(O.interpolate(c, lg), lg + blowup) for c, lg in zip(cols, logs)]
    return ext, O.merkle_root(ext)


@pytest.mark.parametrize("logs,blowup", [([5, 3, 7, 7, 2, 5, 9, 1], 1), ([4, 4, 6], 2), ([10, 1, 12, 3, 12, 8], 1),
                                         ([2], 3)])
@pytest.mark.parametrize("graph", [False, True])
def test_commit_plan_matches_oracle(mod, logs, blowup, graph):
    rng = np.random.default_rng(sum(logs) * 10 + blowup)
    plan = mod.CommitPlan(logs, blowup, use_graph=graph)
    for rep in range(2):  # second run: new inputs (graph replay)
        cols = [rng.integers(0, P, 1 << lg, dtype=np.int64).astype(np.uint32) for lg in logs]
        ext, root = expected(cols, logs, blowup)
        got = plan.run([mod.to_device(c) for c in cols])
        assert got == root
        for i in range(len(logs)):
            assert np.array_equal(plan.extended(i), ext[i])
    plan.close()


def test_commit_plan_layers_and_unaligned_inputs(mod):
    """Layers match a layer-by-layer oracle commit; inputs at odd word offsets
    (not 16-byte aligned) take the eager path of a graph plan."""
    logs, blowup = [6, 4, 6, 3], 1
    rng = np.random.default_rng(3)
    cols = [rng.integers(0, P, 1 << lg, dtype=np.int64).astype(np.uint32) for lg in logs]
    ext, root = expected(cols, logs, blowup)
    plan = mod.CommitPlan(logs, blowup, use_graph=True)
    assert plan.run([mod.to_device(c) for c in cols]) == root
    # oracle layers: sorted by size, injected at their layer
    order = sorted(range(len(logs)), key=lambda i: -logs[i])
    prev = None
    for L in range(max(logs) + blowup, -1, -1):
        inj = [ext[i] for i in order if logs[i] + blowup == L]
        prev = O.commit_on_layer(L, prev, inj)
        assert np.array_equal(plan.layer(L), prev)
    big = [torch.zeros((1 << lg) + 1, dtype=torch.int32, device="cuda") for lg in logs]
    views = []
    for b, c in zip(big, cols):
        b[1:] = mod.to_device(c)
        views.append(b[1:])
    assert plan.run(views) == root
    plan.close()
