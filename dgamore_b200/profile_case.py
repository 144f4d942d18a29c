"""Small profiling case of the ladder pass: a configuration's orbitals and fermionic box (so the BSE matrices
have the full compound size N) on a reduced momentum grid and bosonic box, so that one BSE launch is a single
wave of CTAs and an ncu capture of it holds about a gigabyte of device memory.

    python -m dgamore_b200.profile_case --config c3 --nk 4 --niw 10 --passes 1 [--precision mixed]

Runs the passes and prints one JSON line with the shapes, the number of BSE items and the kernels launched.
With ``--eliashberg K`` it then builds the pairing vertices of the same pass (FP64, three-leg vertex kept) and
applies the singlet gap-equation operator K times.  The full vertex of the pp box comes out of the pass's own
BSE (LadderPass(eliashberg_pp=niv_pp)); ``--separate-vertex`` builds it with the separate kernel instead:

    python -m dgamore_b200.profile_case --config c4_bilayer --nk 48 --niw 30 --eliashberg 5

With ``--local-sde`` it runs the local Schwinger-Dyson equation instead, on inputs made from the model vertex
(synthetic.local_sde_inputs) with the configuration's fermionic box and ``--niw`` bosonic frequencies:

    python -m dgamore_b200.profile_case --config c3 --niw 40 --local-sde --passes 2
"""

from __future__ import annotations

import argparse
import dataclasses
import json

import torch

from . import synthetic
from .pipeline import LadderPass


def reduced_config(name: str, nk: int, niw: int) -> synthetic.DgaConfig:
    cfg = synthetic.CONFIGS[name]
    return dataclasses.replace(cfg, name=f"{name}_nk{nk}_niw{niw}", nk=(nk, nk, 1), niw=niw)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c3")
    ap.add_argument("--nk", type=int, default=4)
    ap.add_argument("--niw", type=int, default=10)
    ap.add_argument("--passes", type=int, default=1)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--eliashberg", type=int, default=0, help="gap-equation operator applications after the pass")
    ap.add_argument("--separate-vertex", action="store_true",
                    help="build the Eliashberg full vertex with its own kernel, not inside the pass's BSE")
    ap.add_argument("--local-sde", action="store_true", help="run the local Schwinger-Dyson equation instead")
    args = ap.parse_args(argv)
    if args.local_sde:
        from .local_sde import LocalSde

        base = synthetic.CONFIGS[args.config]
        lsi, _ = synthetic.local_sde_inputs(base, niw=args.niw)
        sde = LocalSde(*lsi)
        for _ in range(args.passes):
            sde.run()
        torch.cuda.synchronize()
        sde.check()
        print(json.dumps({"case": f"{args.config}_local_niw{args.niw}", "n_orb": sde.n, "N": sde.N, "Nf": sde.Nf,
                          "matrices_per_lu": 2 * sde.W, "passes": args.passes}))
        return
    cfg = reduced_config(args.config, args.nk, args.niw)
    inp = synthetic.make_inputs(cfg)
    fuse = args.eliashberg > 0 and args.precision == "fp64" and not args.separate_vertex
    eli_pp = None
    if fuse:
        from .eliashberg_solver import default_niv_pp

        eli_pp = default_niv_pp(cfg.niw, cfg.niv)
    lp = LadderPass(inp, keep_intermediates=args.eliashberg > 0, precision=args.precision, eliashberg_pp=eli_pp)
    for _ in range(args.passes):
        lp.run()
    torch.cuda.synchronize()
    status = int(lp.bse_status.abs().sum()) + int(lp.status.abs().sum())
    print(json.dumps({
        "case": cfg.name, "n_orb": lp.sh.n_orb, "N": lp.sh.N, "n_q": lp.sh.n_q, "bse_items": lp.n_items,
        "passes": args.passes, "precision": args.precision, "status": status,
        "device_bytes": lp.device_bytes() + (lp.bse_scratch.numel() * 16 if lp.bse_scratch is not None else 0),
    }))
    if status:
        raise SystemExit(f"non-zero status {status}")
    if args.eliashberg > 0:
        from .eliashberg_solver import EliashbergSolver

        es = EliashbergSolver(lp)
        x = torch.ones(es.dim, dtype=torch.complex128, device=lp.dev)
        out = torch.empty_like(x)
        for _ in range(args.eliashberg):
            es.matvec("sing", x, out)
        torch.cuda.synchronize()
        print(json.dumps({"eliashberg_M": es.M, "nk": lp.sh.nk_tot, "matvecs": args.eliashberg, "fused": es.fused,
                          "vertex_status": int(es.vertex_status.abs().sum())}))


if __name__ == "__main__":
    main()
