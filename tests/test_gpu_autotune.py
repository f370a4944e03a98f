"""The autotuner: it measures the compiled shapes on the device, installs the
fastest, and every result stays bit-exact with the tuned shapes."""
import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from benchntt_b200 import workloads as W
from gpu_util import DevBuf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tuned(tmp_path_factory):
    ctx = bn.Context(0)
    path = str(tmp_path_factory.mktemp("tune") / "bntt.tune")
    ctx.autotune(path)
    yield ctx, path
    bn.lib().bntt_autotune_reset()
    ctx.close()


def test_cache_file_lists_a_choice_per_size(tuned):
    _, path = tuned
    lines = open(path).read().splitlines()
    assert lines[0].startswith("bntt-autotune 1 ")
    subs = [l for l in lines if l.startswith("sub ")]
    batch = [l for l in lines if l.startswith("batch ")]
    assert {int(l.split()[1]) for l in subs if l.split()[2] == "0"} == set(range(1, 11))
    assert {int(l.split()[1]) for l in batch} == set(range(1, 11))


def test_cache_round_trip_and_device_check(tuned, tmp_path):
    ctx, path = tuned
    ctx.autotune_load(path)
    bad = tmp_path / "other.tune"
    text = open(path).read().splitlines()
    text[0] = "bntt-autotune 1 some_other_gpu|sms=1"
    bad.write_text("\n".join(text) + "\n")
    with pytest.raises(bn.BnttError) as e:
        ctx.autotune_load(str(bad))
    assert e.value.status == bn.EINVAL


@pytest.mark.parametrize("logn", [3, 6, 10, 14, 20])
def test_tuned_plans_bit_exact(tuned, logn):
    ctx, _ = tuned
    n = 1 << logn
    batch = max(1, (1 << 14) >> logn)
    x = C.uniform_pairs(3 + logn, n * batch, C.Q_NTT)
    t = C.uniform_pairs(4 + logn, n, C.Q_NTT)
    plan = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    y = np.empty_like(x)
    plan.forward(y, x)
    assert np.array_equal(y, C.oracle_ntt(x, t, logn, threads=8, form=1))
    plan.close()


def test_tuned_batch_bit_exact(tuned):
    ctx, _ = tuned
    b = W.uneven_batch(seed=9, n_small=4000, large=((16, 1), (20, 1)))
    tables = {n: C.uniform_pairs(W.SEED_TWIDDLE_BASE + n, 1 << n, C.Q_NTT) for n in b.sizes}
    plans = {n: bn.Plan(ctx, n, C.Q_NTT, C.MU_NTT, tables[n]) for n in b.sizes}
    pid = {n: i for i, n in enumerate(b.sizes)}
    eng = bn.Batch(ctx, [plans[n] for n in b.sizes])
    x = C.uniform_pairs(W.SEED_INPUT, b.total, C.Q_NTT)
    dx, dy = DevBuf.from_array(ctx, x), DevBuf(ctx, b.total * 16)
    offs = [16 * int(o) for o in b.offsets]
    eng.run_dev(bn.Batch.jobs([dx.addr + o for o in offs], [dy.addr + o for o in offs],
                              [pid[int(n)] for n in b.logns]))
    assert eng.status() == bn.OK
    xs = [x[o:o + (1 << n)] for o, n in zip(b.offsets, b.logns)]
    want = np.concatenate(C.oracle_ntt_jobs(xs, [tables[int(n)] for n in b.logns],
                                            [int(n) for n in b.logns], threads=8))
    assert np.array_equal(dy.to_array(b.total), want)
    dx.free()
    dy.free()
    eng.close()
    for p in plans.values():
        p.close()
