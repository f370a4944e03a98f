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


def _force(ctx, tmp_path, head: str, lines: list[str]):
    """Installs exactly the given tuner choices (a hand-written tune file)."""
    f = tmp_path / "forced.tune"
    f.write_text(head + "".join(l + "\n" for l in lines))
    bn.lib().bntt_autotune_reset()
    ctx.autotune_load(str(f))


# (log2n, logr, tpc, minb, src): the staged kernels (inputs staged into
# shared memory a tile ahead; src=3 also holds the table there) at 4 and 5
# resident CTAs per SM, the 48-register plain shapes and 8 elements per thread
# at 2^4
SHAPES = ([(m, 2, 1024 >> m, 4, src) for m in range(3, 11) for src in (1, 3)] +
          [(m, 2, 1024 >> m, 5, src) for m in range(3, 9) for src in (0, 1, 3)] +
          [(4, 3, 128, 4, 0)])


@pytest.mark.parametrize("logn,logr,tpc,minb,src", SHAPES, ids=lambda v: str(v))
def test_candidate_shapes_bit_exact(tuned, tmp_path, logn, logr, tpc, minb, src):
    """Every small-transform candidate the tuner can pick, forced through a
    tune file: more tiles than CTAs (for staged kernels the copy of the next
    tile overlaps the current one) and a partial last tile, against the
    oracle."""
    ctx, path = tuned
    head = open(path).readline()
    _force(ctx, tmp_path, head, [f"sub {logn} 0 1 {logr} {tpc} {minb} {src}"])
    n = 1 << logn
    batch = (2 * minb * ctx.sm_count + 5) * tpc + 3
    x = C.uniform_pairs(40 + logn, n * batch, C.Q_NTT)
    t = C.uniform_pairs(41 + logn, n, C.Q_NTT)
    plan = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    y = np.empty_like(x)
    plan.forward(y, x)
    assert np.array_equal(y, C.oracle_ntt(x, t, logn, threads=8))
    plan.close()
    ctx.autotune_load(path)   # the measured choices again, for the other tests


@pytest.mark.parametrize("src", [1, 3])
def test_staged_fused_product_and_u128_layout(tuned, tmp_path, src):
    """The staged kernels with the fused pointwise product and with native
    uint128_t buffers."""
    import torch
    ctx, path = tuned
    head = open(path).readline()
    _force(ctx, tmp_path, head, [f"sub 7 0 1 2 8 4 {src}"])
    logn, n, batch = 7, 128, 5001
    x = C.uniform_pairs(51, n * batch, C.Q_NTT)
    b = C.uniform_pairs(52, n * batch, C.Q_NTT)
    t = C.uniform_pairs(53, n, C.Q_NTT)
    plan = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    dx = torch.from_numpy(x.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dy = torch.empty_like(dx)
    plan.forward_mul(dy, dx, db, True, batch)
    torch.cuda.synchronize()
    want = C.oracle_blas("vvmul", C.oracle_ntt(x, t, logn, threads=8), b, C.Q_NTT, C.MU_NTT)
    assert np.array_equal(dy.cpu().numpy().view(np.uint64), want)
    plan.close()
    # the same transform on native little-endian uint128_t buffers
    plan = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, np.ascontiguousarray(t[:, ::-1]), layout=bn.LAYOUT_U128)
    xu = np.ascontiguousarray(x[:, ::-1])
    yu = np.empty_like(xu)
    plan.forward(yu, xu)
    assert np.array_equal(yu[:, ::-1], C.oracle_ntt(x, t, logn, threads=8))
    plan.close()
    ctx.autotune_load(path)
