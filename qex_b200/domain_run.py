"""A CG solve decomposed along t, one rank per GPU (NCCL), under torchrun:

  python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 \
      -m qex_b200.domain_run --dims 32,32,32,64 [--zranks Rz]

Each rank builds the same synthetic fat+Naik field and source (seeded),
keeps its slab, rank 0 makes the NCCL id and broadcasts it over the
torch.distributed process group (gloo), and all ranks solve
stagD2ee(m^2) y = b with qexstag_domain_solveEE.  Rank 0 prints one JSON
line with the iterations, the true residual and the time.
"""
from __future__ import annotations

import argparse
import json
import os


def main():
    import torch
    import torch.distributed as dist
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", default="16,16,16,32")
    ap.add_argument("--mass", type=float, default=0.05)
    ap.add_argument("--r2req", type=float, default=1e-20)
    ap.add_argument("--zranks", type=int, default=0,
                    help="split along t and z with this many ranks along z (0: along t only)")
    a = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from . import domain as DD
    from . import fields as F
    from . import stag as S
    S.init(local)
    dims = tuple(int(v) for v in a.dims.split(","))
    obj = [DD.nccl_unique_id() if rank == 0 else None]
    dist.broadcast_object_list(obj, src=0)
    grid = (a.zranks, world // a.zranks) if a.zranks > 0 else None
    d = DD.DomainSet(dims, world, 8, ranks=[rank], nccl_id=obj[0], grid=grid, device=local)
    g = F.fat_naik_links(dims, 21)
    b = F.even_source(dims, 31)
    d.set_links(g)
    x = b * 0
    sp = S.SolverParams(r2req=a.r2req)
    d.solveEE(x, b, a.mass, sp)
    dist.barrier()
    if rank == 0:
        print(json.dumps({"dims": dims, "ranks": world, "iterations": sp.iterations, "true_r2": sp.r2,
                          "seconds": sp.seconds, "status": sp.status}))
    del d
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
