"""Full sweep of the solver's division against IEEE division on the current GPU: every divisor
significand (2^23) against every numerator significand (2^23) through
pxb_check_quotient_significands, then the seeded random constraints of pxb_check_quotients.

    python -m physxcoopa_b200.check_division [--device N]

Prints one line per 2^20 divisors and a summary; exits 1 on any mismatch. Takes a few minutes.
"""
import argparse
import sys
import time

from . import runtime as R


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    ctx = R.Context(args.device)
    t0 = time.perf_counter()
    total = 0
    step = 1 << 20
    for first in range(0, 1 << 23, step):
        bad = ctx.check_quotient_significands(first, step)
        total += bad
        print(f"divisor significands [{first:#08x}, {first + step:#08x}): {bad} mismatches", flush=True)
    rcp_bad, q_bad = ctx.check_quotients(1 << 32, 7)
    ctx.close()
    print(f"all 2^46 significand pairs: {total} mismatches; refined reciprocal: {rcp_bad} significands off; "
          f"2^32 random constraints: {q_bad} quotients off; {time.perf_counter() - t0:.1f} s")
    return 1 if (total or rcp_bad or q_bad) else 0


if __name__ == "__main__":
    sys.exit(main())
