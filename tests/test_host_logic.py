"""Host-side logic that needs no GPU: cost-aware cluster sizes, the autotuner's candidate splits,
choice and cache, the warm start's canvas and normalisation, the network's layer table, the
large configuration."""
import json
import os

import numpy as np
import pytest


class _FakeBatch:
    def __init__(self, n):
        self.n = n
        self.sizes = {}

    def set_cluster_size(self, c, k):
        self.sizes[c] = k


def test_balance_clusters_keeps_total_and_favours_expensive_cases(pkg):
    its = np.array([244654, 100000, 90000, 150000, 120000, 80000, 110000, 95000,
                    130000, 105000, 90000, 85000, 99000, 140000, 160000, 102000])
    f = _FakeBatch(len(its))
    k = pkg.Batch.balance_clusters(f, its, 192)
    assert k.sum() == 192 and k.min() >= 1 and k.max() <= 16
    assert k[0] == k.max()                                   # the slowest case gets the most CTAs
    assert (its / k).max() < (its / 12).max()                # the heaviest load per CTA goes down
    assert f.sizes == {c: int(k[c]) for c in range(len(its))}
    # more slots than 16 per case can use: everyone capped at 16
    assert (pkg.Batch.balance_clusters(_FakeBatch(4), [1, 2, 3, 4], 1000) == 16).all()
    # fewer slots than cases: one CTA each at least
    assert (pkg.Batch.balance_clusters(_FakeBatch(5), [5, 1, 1, 1, 1], 3) >= 1).all()


def test_autotune_fill_candidates(pkg):
    from importlib import import_module
    at = import_module(pkg.__name__ + ".autotune")
    items, _ = pkg.configs.cfg_batch(16, seed=101, sizes=(153,))
    c1 = at.fill_candidates(items, 148, 1)
    nodes = 154 * 154
    # 16 cases on 148 SMs: one wave at 148 // 16 = 9 CTAs per case, and the neighbours 8 and 10
    assert sorted(-(-nodes // npc) for npc in c1) == [8, 9, 10]
    assert at.fill_candidates(items, 0, 1) == []
    assert at.signature(items) == at.signature(list(reversed(items)))


def test_canvas_and_node_count(pkg):
    from importlib import import_module
    ws = import_module(pkg.__name__ + ".warmstart")
    assert ws.canvas_for(153, 153) == (160, 160)
    assert ws.canvas_for(24, 24) == (32, 32)
    assert ws.canvas_for(100, 50) == (56, 104)
    nx, ny = 7, 5
    assert ws.valid_nodes(nx, ny) == (nx + 1) * ny + nx * (ny + 1) + 3 * nx * ny


def test_normalizer_from_samples(pkg):
    from importlib import import_module
    ws = import_module(pkg.__name__ + ".warmstart")
    rng = np.random.default_rng(0)
    X = rng.standard_normal((3, 8, 8, 11)) * 4.0 + 2.0
    T = rng.standard_normal((3, 8, 8, 8)) * 0.5
    Wt = np.zeros((3, 8, 8, 8))
    Wt[..., :5] = 1.0
    Wt[:, 6:, :, :] = 0.0                                   # rows outside the case
    n = ws.Normalizer.from_samples(X, T, Wt, device="cpu")
    m = Wt[..., 0] > 0
    assert np.allclose(n.in_shift.numpy()[0], X[..., 0][m].mean(), rtol=1e-5)
    assert np.allclose(n.in_mul.numpy()[0], 1.0 / X[..., 0][m].std(), rtol=1e-5)
    assert n.in_shift.numpy()[5] == 0.0 and n.in_mul.numpy()[5] == 1.0   # porous indicator untouched
    osc = n.out_scale.numpy()
    assert osc.shape == (16,) and np.allclose(osc[0], np.sqrt(np.mean(T[..., 0][m] ** 2)), rtol=1e-5)
    assert (osc[5:8] == 1.0).all() and (osc[8:] == 1.0).all()   # padding channels, increment weights
    d = n.to_dict()
    assert set(d) == {"in_shift", "in_mul", "out_scale", "inc_weight", "smooth"}


def test_layer_table_and_flops(pkg):
    from importlib import import_module
    un = import_module(pkg.__name__ + ".unet")
    convs, n = un.layer_table()
    names = [L.name for L in convs]
    assert names[:2] == ["enc0a", "enc0b"] and names[-1] == "head" and len(convs) == 15
    ends = 0
    for L in convs:
        assert L.off_w % 64 == 0 and L.off_w >= ends       # 16-byte aligned BF16 slices, no overlap
        assert L.kp % 8 == 0 and L.kp >= 9 * L.cin
        ends = L.off_b + L.cout
    assert n >= ends and n == 1951808
    # 2 * 9 * Cin * Cout * pixels summed over the layers (head at its 5 real channels)
    assert un.conv_flops(160, 160) == 8493465600


def test_large_configuration(pkg):
    prm, mesh, st, itc, n = pkg.configs.cfg_large(64, 32)
    assert (prm.imax, prm.jmax, n, itc) == (64, 32, 1000, 1)
    flag = mesh["flag"] != 0
    left, right = flag[:32].any(), flag[32:].any()
    assert left and right and not flag[30:34].any()         # two separate blocks
    assert prm.Re == 400.0 and prm.solve_scalars == 1


class _FakeTunePkg:
    """Stands in for the library in the autotuner: a batch whose 'run' reports many pseudo-
    iterations for one launch shape only, so that shape must win."""
    ARITH_FAST = 1
    OPT_THREADS, OPT_CTAS_PER_SM, OPT_NODES_PER_CTA, OPT_L1_LOADS, OPT_STAGED, OPT_ENGINE = range(1, 7)
    WIN = {1: 512, 2: 1, 3: 1024, 5: 1, 6: 0}

    def __init__(self):
        self.batches = 0
        pkg = self

        class Batch:
            def __init__(self, params, meshes):
                pkg.batches += 1
                self.n, self.opt = len(params), {}

            def set_option(self, k, v):
                self.opt[k] = v

            def set_state(self, c, st):
                pass

            def run(self, steps, itc):
                win = all(self.opt.get(k) == v for k, v in pkg.WIN.items())
                return None, np.full((self.n, 1), 1000 if win else 10), None, None

            def close(self):
                pass

        self.Batch = Batch


def test_autotune_picks_fastest_and_caches_atomically(pkg, tmp_path, monkeypatch):
    from importlib import import_module
    at = import_module(pkg.__name__ + ".autotune")
    monkeypatch.setattr(at, "CACHE_DIR", str(tmp_path))
    items, _ = pkg.configs.cfg_batch(3, seed=5, sizes=(51,))
    fake = _FakeTunePkg()
    best = at.tune(fake, items, iters=20)
    assert best == {"threads": 512, "ctas_per_sm": 1, "nodes_per_cta": 1024, "staged": 1, "engine": 0}
    files = os.listdir(tmp_path)
    assert len(files) == 1 and files[0].endswith(".json")          # no temporary file left behind
    with open(os.path.join(tmp_path, files[0])) as f:
        entry = json.load(f)
    n_cand = sum(len(set(at.NODES)) * (2 if per_sm == 1 else 1) for _, per_sm in at.SHAPES) + 1
    assert entry["best"] == best and len(entry["table"]) == n_cand   # no SMs visible: fixed candidates
    assert at.tune(fake, items) == best and fake.batches == 1         # second call: from the cache
    with open(os.path.join(tmp_path, files[0]), "w") as f:
        f.write('{"key": "trunc')                                     # a partial entry is re-tuned
    assert at.tune(fake, items, iters=20) == best and fake.batches == 2


def test_step_log_records(pkg, tmp_path):
    from importlib import import_module
    ws = import_module(pkg.__name__ + ".warmstart")
    path = tmp_path / "steps.jsonl"
    log = ws.StepLog(str(path), label="learned")
    res0 = np.array([[3e-3, 1e-3, 5e-4], [2e-3, 4e-3, np.nan]])
    log.write(4, np.array([120, 7]), np.array([9.5e-7, 8.1e-7]), status=np.array([1, 2]),
              chosen=np.array([2, 0]), res0=res0)
    log.write(5, np.array([90, 1]), np.array([9.9e-7, np.nan]))       # a plain step: no start fields
    log.close()
    lines = [json.loads(x) for x in path.read_text().splitlines()]
    assert len(lines) == 4
    assert lines[0] == {"step": 4, "case": 0, "pseudo_iterations": 120, "error": 9.5e-7, "run": "learned",
                        "status": "done", "start": "learned",
                        "initial_residual": {"plain": 3e-3, "extrap": 1e-3, "learned": 5e-4}}
    assert lines[1]["status"] == "failed" and lines[1]["start"] == "plain"
    assert lines[1]["initial_residual"]["learned"] is None                 # candidate not built
    assert lines[2]["step"] == 5 and "start" not in lines[2] and "status" not in lines[2]
    assert lines[3]["error"] != lines[3]["error"]                           # NaN error kept as NaN


def test_eval_only_refuses_the_learned_mode(pkg):
    from importlib import import_module
    tw = import_module(pkg.__name__ + ".train_warmstart")
    with pytest.raises(SystemExit, match="plain,extrap"):
        tw.main(["--eval-only", "--n", "24", "--modes", "plain,extrap,learned"])
