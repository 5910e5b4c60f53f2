"""One rank of the row-sharded pipeline, run as its own process (test
infrastructure for test_gpu_shard_mp.py; bench.py's multi-GPU arm uses the
same calls).

    python tests/shard_worker.py <input dir> <host|device> <out.npz>

RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT come from the environment;
the process group is gloo (CPU and CUDA tensors), with a short timeout so
that a rank that never joins ends the others with an error.  Every rank
runs ald_kappa_pipeline_sharded(_dev) on its own context; rank 0 writes the
results.
"""
import datetime
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "anharmonic-lattice-dynamics_b200", "python"))


def main():
    d, mode, out = sys.argv[1], sys.argv[2], sys.argv[3]
    import torch
    import torch.distributed as dist

    import ald
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ctx = ald.Context(d)
        dev = mode == "device"
        gather = ald.torch_allgather_device() if dev else ald.torch_allgather()
        if dev:  # the exchange runs on a torch stream that the library also uses
            st = torch.cuda.Stream()
            ctx.set_stream(st.cuda_stream)
        res = ctx.kappa_pipeline_sharded(rank, world, gather, device=dev)
        torch.cuda.synchronize()
        if rank == 0:
            np.savez(out, **{k: np.asarray(v) for k, v in res.items() if k not in ("stage_ms", "launches")})
        ctx.close()
    finally:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
