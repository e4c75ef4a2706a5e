"""Seeded realizations of one workload with the realization passes' choices given on the
command line instead of measured planning, so that a profiler sees only the FP64 spectrum
and the realization passes of each choice, in order.

Each `--run` is one plan: a list of PASS=VARIANT[:CTAS] entries (pass 0 noise, 1 middle
strided, 2 complex-to-real; variant 0 paired FP32, 1 scalar, 2 staged tiles -- TMA for pass 1,
bulk copies for pass 2; CTAS resident CTAs per SM, 0 = as many as fit) and optionally
G=<plane groups>.  Passes not named take variant 0 at full occupancy.

  python parafields-core_b200/pass_profile.py --cells 256 256 256 --covariance matern32 \\
      --corr-length 0.2 0.1 0.05 --approximate --run 2=0 --run 2=2 --realizations 2

With --matvec K the plan instead runs K FP32 matvecs on FP32 device vectors (the CG's inner
products run the same kernels with FP64 vectors in and out), e.g. the 128^3 covariance-inverse workload with a geometric anisotropy:

  python parafields-core_b200/pass_profile.py --cells 128 128 128 --covariance exponential \\
      --corr-length <9 values of the matrix> --approximate --matvec 2
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import pfb200  # noqa: E402


def wisdom_lines(info, choices, groups):
    """wisdom text fixing every pass of the plan (keys as the library's measured planning)"""
    dim = info.dim
    T = [info.ext_cells[i] for i in range(3)]
    n = [info.cells[i] for i in range(3)]
    t0c = T[0] // 2 + 1
    prec = info.precision
    keys = {0: (T[dim - 1], t0c, T[1] if dim == 3 else 1),
            2: (T[0], n[1] * n[2] if dim == 3 else n[1], 1)}
    if dim == 3:
        keys[1] = (T[1], t0c, n[2])
    lines = []
    for p, (L, np_, nouter) in sorted(keys.items()):
        v, c = choices.get(p, (0, 0))
        lines.append("%d %d %d %d %d %d %d" % (p, L, np_, nouter, prec, v, c))
    L, np_, nouter = keys[0]
    lines.append("3 %d %d %d %d 0 %d" % (L, np_, nouter, prec, groups))
    return "\n".join(lines) + "\n"


def parse_run(text):
    choices, groups = {}, 1
    for item in text.split(","):
        k, v = item.split("=")
        if k.strip().upper() == "G":
            groups = int(v)
            continue
        var, _, cap = v.partition(":")
        choices[int(k)] = (int(var), int(cap or 0))
    return choices, groups


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--cells", type=int, nargs="+", default=[256, 256, 256])
    ap.add_argument("--covariance", default="matern32")
    ap.add_argument("--corr-length", type=float, nargs="+", default=[0.2, 0.1, 0.05])
    ap.add_argument("--approximate", action="store_true")
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--run", action="append", default=[], help="PASS=VARIANT[:CTAS],...[,G=groups]")
    ap.add_argument("--realizations", type=int, default=2)
    ap.add_argument("--matvec", type=int, default=0,
                    help="instead of realizations: this many FP32 matvecs (C x) on FP32 device vectors")
    a = ap.parse_args(argv)
    import torch

    dim = len(a.cells)
    d = pfb200.make_desc(dim=dim, cells=a.cells, covariance=a.covariance, corr_length=a.corr_length,
                         approximate=a.approximate, precision=pfb200.PREC_F64 if a.fp64 else pfb200.PREC_F32)
    if a.matvec:
        P = pfb200.Plan(d)
        P.spectrum_build()
        n = P.info.domain_size
        x = torch.randn(n, dtype=torch.float32, device="cuda")
        y = torch.empty_like(x)
        for _ in range(a.matvec):
            P.matvec(x, op=pfb200.OP_MUL, precision=pfb200.PREC_F32, out=y)
        torch.cuda.synchronize()
        print("%d matvecs" % a.matvec, flush=True)
        P.close()
        return
    for run in a.run or ["0=0"]:
        choices, groups = parse_run(run)
        P = pfb200.Plan(d)
        pfb200.wisdom_forget()
        pfb200.wisdom_import(wisdom_lines(P.info, choices, groups))
        P.spectrum_build()
        if P.autotune() is not False:
            raise RuntimeError("the pass choices did not cover the plan")
        out = torch.empty(P.info.domain_size, dtype=torch.float64 if a.fp64 else torch.float32, device="cuda")
        for r in range(a.realizations):
            P.generate(seed=r + 1, out=out)
        torch.cuda.synchronize()
        print("run %s: %d realizations" % (run, a.realizations), flush=True)
        P.close()
    pfb200.wisdom_forget()


if __name__ == "__main__":
    main()
