"""Generate the committed golden fixtures from the reference's own code.

Run in a container that has the reference tree (given as the argument, or
$COMPLAB_REFERENCE, or BASELINE.json's reference_path) and the compiled
oracle/_ref/libref.so (``make -C oracle``):

    python tests/golden/make_golden.py [REFERENCE_ROOT]

Writes tests/golden/*.npz:
  surrogate_shipped.npz  the trained network shipped in surrogateModel.hh
                         (weights parsed from the header text) and the
                         reference's defineSurrogateModel output on 512 inputs
                         spread over its training box (the compile-and-compare
                         check of surrogate_training/verifyExport.py:61-131).
  speciation_pcf.npz     the reference's PCF+Anderson solver (tol 1e-10, 200
                         iterations, depth 4) on example 04's carbonate tableau
                         and on 5x14 random-tableau samples.
The GPU tests read only these files; nothing at test time reads the reference.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def parse_shipped_net(ref_root):
    text = open(os.path.join(ref_root, "surrogateModel.hh")).read()

    def vec(name):
        m = re.search(r"static const std::vector<double> %s\s*=\s*\{([^}]*)\}" % name, text)
        return np.array([float(v) for v in m.group(1).split(",")])

    def mat(name):
        m = re.search(r"static const std::vector<std::vector<double>> %s\s*=\s*\{(.*?)\};" % name, text, re.S)
        rows = re.findall(r"\{([^{}]*)\}", m.group(1))
        return np.array([[float(v) for v in r.split(",")] for r in rows])

    def scal(name):
        m = re.search(r"static const double %s\s*=\s*([-0-9.eE+]+);" % name, text)
        return float(m.group(1))

    W = [mat("IW1_1"), mat("LW2_1"), mat("LW3_2"), mat("LW4_3"), vec("LW5_4").reshape(1, -1)]
    b = [vec("b1"), vec("b2"), vec("b3"), vec("b4"), np.array([scal("b5")])]
    scaling = dict(x_offset=[scal("x_offset0"), scal("x_offset1")], x_gain=[scal("x_gain0"), scal("x_gain1")],
                   x_ymin=scal("x_ymin"), y_ymin=scal("y_ymin"), y_gain=scal("y_gain"), y_offset=scal("y_offset"))
    return W, b, scaling


def main():
    from oracle import oracle as o
    from conftest import load_workloads, reference_root
    ref_root = sys.argv[1] if len(sys.argv) > 1 else reference_root()
    if not ref_root:
        raise SystemExit("no reference tree: pass its path or set COMPLAB_REFERENCE")
    wl = load_workloads()
    if o.ref_lib() is None:
        raise SystemExit("build oracle/_ref first: make -C oracle")
    # ---- surrogate
    W, b, sc = parse_shipped_net(ref_root)
    rng = np.random.default_rng(2024)
    lo = np.array(sc["x_offset"])
    hi = lo + 2.0 / np.array(sc["x_gain"])
    fin = lo + (hi - lo) * rng.random((512, 2))
    bior = o.ref_surrogate(fin)
    flat = {"W%d" % l: W[l] for l in range(5)}
    flat.update({"b%d" % l: b[l] for l in range(5)})
    np.savez(os.path.join(HERE, "surrogate_shipped.npz"), fin=fin, bior=bior,
             x_offset=np.array(sc["x_offset"]), x_gain=np.array(sc["x_gain"]), x_ymin=sc["x_ymin"],
             y_ymin=sc["y_ymin"], y_gain=sc["y_gain"], y_offset=sc["y_offset"], **flat)
    # ---- speciation
    S4 = np.array([[1, 0], [0, 1], [1, -1], [1, 1]], float)
    lk4 = np.array([0.0, 0.0, -10.33, 6.35])
    sp4 = np.array([[1e-3, 1e-7, 1e-30, 1e-30], [5e-3, 1e-8, 1e-30, 1e-30], [2e-4, 3e-6, 1e-30, 1e-30]])
    out4, it4, cv4 = o.ref_pcf_solve(S4, lk4, [0, 1], sp4)
    S, logk, cs = wl.tableau(5, 9, seed=4)
    T, xs, cstar, acc = wl.speciation_batch(S, logk, 256, seed=77)
    out, it, cv = o.ref_pcf_solve(S, logk, cs, cstar)
    np.savez(os.path.join(HERE, "speciation_pcf.npz"), S4=S4, logk4=lk4, species4=sp4, out4=out4, it4=it4,
             cv4=cv4, S=S, logk=logk, comp_species=np.array(cs), totals=T, xstar=xs, cstar=cstar, pcf_out=out,
             pcf_it=it, pcf_cv=cv, acceptance=acc)
    print("wrote fixtures; PCF converged %d/%d on the 5x14 samples" % (int(cv.sum()), cv.size))


if __name__ == "__main__":
    main()
