"""bench.py's multi-GPU path (--gpus N under torch.distributed.run) run as
N processes sharing one GPU: the process group is gloo, so the halos are
staged through pinned host memory and no kernel waits on another process's
(NCCL ranks must each have their own GPU).  Everything else -- the block
decomposition, the per-stage exchange, the timing with a barrier and the
maximum over ranks, the end-to-end leg, the one JSON line from rank 0 -- is
the code the N-GPU run executes."""
import pytest

from tests.test_bench_contract import torchrun_bench

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nproc,dims,par", [(2, "", "blocks2x1x1"), (4, "2,2,1", "blocks2x2x1")])
def test_bench_multi_rank_line(cuda, nproc, dims, par):
    args = ["--gpus", str(nproc), "--backend", "gloo", "--steps", "3", "--warmup", "3",
            "--nx", "64", "--ny", "32", "--nz", "32"]
    if dims:
        args += ["--dims", dims]
    lines, err = torchrun_bench(nproc, *args)
    assert len(lines) == 1, err[-2000:]
    d = lines[0]
    assert d["n_gpus"] == nproc and d["steps"] == 3 and d["warmup"] == 3
    assert d["scaling"] == "weak" and d["value"] > 0 and d["device_status"] == 0
    c = d["config"]
    assert c["parallelism"] == par and c["grid_per_gpu"] == [64, 32, 32]
    assert d["halo_transport"].startswith("gloo")
    px, py, pz = (int(v) for v in (dims or f"{nproc},1,1").split(","))
    assert c["grid"] == [64 * px, 32 * py, 32 * pz]
    assert d["e2e"]["value"] > 0 and d["gpu_launches"] > 0
