"""Write tests/golden/oracle_regression.json: SHA-256 digests and sums of
the oracle's state after four steps of each seeded deck below.

The reference has no golden files and no Fortran compiler exists here, so
these fixtures pin the oracle against itself: a later change to the C++
restatement that alters any bit of any field shows up in
tests/test_golden_cpu.py.  Regenerate only for an intended change, and say
why in the commit.

    python tests/golden/make_oracle_regression.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

STATE = ["rho", "energy", "vx", "vy", "vz", "bx", "by", "bz"]
STEPS = 4


def cases():
    from lare3d_b200 import decks
    from lare3d_b200.abi import BC_USER, EOS_PI
    return {
        "blast_12": lambda: decks.blast(12),
        "blast_12_user_x": lambda: decks.blast(12, xbc_min=BC_USER, xbc_max=BC_USER),
        "orszag_tang_12": lambda: decks.orszag_tang(12),
        "open_blast_12": lambda: decks.open_blast(12),
        "conduction_10": lambda: decks.conduction(10, kappa_0=1.0e-4),
        "partially_ionised_10": lambda: decks.partially_ionised(10, eta_bar=1e-2),
        "partially_ionised_pi_10": lambda: decks.partially_ionised(10, eos_number=EOS_PI, cowling=False),
        "radiative_blast_10": lambda: decks.radiative_blast(10),
        "orszag_tang_10_rke_cooling": lambda: decks.orszag_tang(10, rke=1, cooling_term=1),
    }


def run(make):
    from oracle import oracle
    d = make()
    s = oracle.simulation(d)
    s.start(d.state)
    for k in range(1, STEPS + 1):
        s.step(k)
    st = s.download()
    out = {}
    for f in STATE:
        a = st[f]
        out[f] = {"sha256": hashlib.sha256(a.tobytes(order="F")).hexdigest(), "sum": float(a.sum()),
                  "sumsq": float((a * a).sum())}
    sc = s.scalars()
    out["_scalars"] = {"time": sc.time, "dt": sc.dt}
    s.close()
    return out


def main():
    res = {"steps": STEPS, "cases": {name: run(make) for name, make in cases().items()}}
    with open(os.path.join(HERE, "oracle_regression.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
