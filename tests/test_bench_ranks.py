"""The bench on CPU: two gloo ranks aggregate their timings (max of the times, sum of the
walker-steps), the reference arm under torchrun runs on rank 0 only, and the learned-proposal
arm trains on an engine of its own."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t, k, ws = bench.aggregate_ranks(dist, 100.0 + 50.0 * rank, 90.0 + 10.0 * rank, 2048 + rank)
    out[rank] = (t, k, ws)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_aggregate_max_time_and_total_work():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        assert out[r] == (150.0, 100.0, 4097.0)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_harness")),
                    reason="reference harness not built")
def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] == "reference"


def test_learned_arm_trains_on_a_separate_engine():
    """The VN comparison's learned arm: the network trains on its own engine (grid walk from the
    start, then closed) and only its parameters reach the measured engine, which has not walked."""
    import argparse
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    from mpsqmc_b200.capi import OPT_PROPOSAL, OPT_PROPOSAL_TRAINING, PROPOSAL_LEARNED

    made = []

    class Fake:
        def __init__(self):
            self.opts, self.steps, self.closed, self.params = {}, 0, False, None
            made.append(self)

        def set_option(self, k, v):
            self.opts[k] = v

        def set_rng(self, seed, skip):
            self.seed = seed

        def walk(self, n):
            self.steps += n
            return [{"n_walkers": 4}] * n

        def proposal_stats(self):
            return {"updates": self.steps, "loss": 0.5}

        def proposal_params(self, p=None):
            if p is None:
                return np.full(3, float(len(made)))
            self.params = p

        def close(self):
            self.closed = True

    args = argparse.Namespace(proposal="learned", train_steps=7, workspace="auto", canon=None, precision="tf32x3",
                              proposal_mix=None)
    measured = Fake()
    params, info = bench.train_proposal(Fake, args, 0, 11)
    bench.use_proposal(measured, params)
    trainer = made[1]
    assert trainer is not measured and trainer.closed and trainer.steps == 7
    assert trainer.opts[OPT_PROPOSAL_TRAINING] == 1
    assert measured.steps == 0 and measured.opts[OPT_PROPOSAL] == PROPOSAL_LEARNED
    np.testing.assert_array_equal(measured.params, params)
    assert info["adam_steps"] == 7 and info["pairs"] == 28
    args.proposal = "grid"
    assert bench.train_proposal(Fake, args, 0, 11) == (None, None)
