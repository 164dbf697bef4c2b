"""Times the MPM step on the mudflow workload, per kernel class.

    python -m amsc_b200.profile_step [N] [K] [W]

Builds the N x N mudflow (hx = 0.5 m, same shapes as the 2048 x 2048
benchmark scaled by N/2048), runs W warm-up steps (default 3) and K timed
steps (default 20), and prints milliseconds per step for the sort, P2G, G2P
and the remaining kernels (CUDA events on the library stream).  Meant as the
command to run under a profiler; a large W profiles the flow after it has
piled up.
"""
import sys

from . import scenarios
from .dampm import Solver


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    N = int(argv[0]) if argv else 2048
    K = int(argv[1]) if len(argv) > 1 else 20
    W = int(argv[2]) if len(argv) > 2 else 3
    d = scenarios.mudflow(N=N)
    with Solver(d) as s:
        s.step(W)
        s.sync()
        s.timings(True)
        s.step(K)
        tm = s.timings(False)
        st = s.status()
        print(f"np {st['np']} it {st['it']} t {st['t']:.6g} dt {st['dt']:.6g}")
        print("ms per step: sort %.4f p2g %.4f g2p %.4f other %.4f total %.4f"
              % tuple(tm / K))
        print("particle-steps/s %.4e" % (st["np"] * K / (tm[4] * 1e-3)))
        print("launches", s.last_launch_count())


if __name__ == "__main__":
    main()
