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
  uranium_tableau.npz    the 17-component x 95-species tableau of the
                         reference's uranium example (its <equilibrium> block),
                         64 known-answer samples, and the reference's PCF +
                         Anderson solve of each from its known species and
                         from its cold vector (components at their totals).
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


def parse_uranium_tableau(ref_root):
    """The <equilibrium> block of the reference's uranium example: 17
    components over 95 species (stoichiometry rows species0..species94 and
    their logK), and for each component the species whose row is its unit
    vector."""
    text = open(os.path.join(ref_root, "CompLaB_example_uranium_zhao.xml")).read()
    block = re.search(r"<equilibrium>(.*?)</equilibrium>", text, re.S).group(1)
    comps = re.search(r"<components>([^<]*)</components>", block).group(1).split()
    sto = re.search(r"<stoichiometry>(.*?)</stoichiometry>", block, re.S).group(1)
    lk = re.search(r"<logK>(.*?)</logK>", block, re.S).group(1)
    rows = {int(i): [float(v) for v in body.split()] for i, body in re.findall(r"<species(\d+)>([^<]*)</species\1>", sto)}
    ks = {int(i): float(v) for i, v in re.findall(r"<species(\d+)>\s*([-0-9.eE+]+)\s*</species\1>", lk)}
    ns, nc = len(rows), len(comps)
    S = np.array([rows[i] for i in range(ns)])
    logk = np.array([ks.get(i, 0.0) for i in range(ns)])
    assert S.shape == (ns, nc)
    cs = []
    for j in range(nc):
        e = np.zeros(nc); e[j] = 1.0
        hit = [i for i in range(ns) if np.array_equal(S[i], e)]
        cs.append(hit[0] if hit else -1)
    return S, logk, cs, comps


def uranium_samples(S, logk, n, seed):
    """Known answers for the uranium tableau: free-component logs drawn per
    component (H+ 1e-9..1e-5, the others 1e-8..1e-3), species formed from them,
    totals T = S^T c; kept where no species leaves [1e-30, 10^0.5] and every
    total is positive."""
    rng = np.random.default_rng(seed)
    ns, nc = S.shape
    keep_x, keep_c, keep_T = [], [], []
    while sum(len(k) for k in keep_x) < n:
        x = rng.uniform(-8.0, -3.0, (4096, nc))
        x[:, 0] = rng.uniform(-9.0, -5.0, 4096)
        lc = logk[None, :] + x @ S.T
        active = np.abs(S).sum(1) > 0
        ok = ((lc[:, active] <= 0.5) & (lc[:, active] >= -30)).all(1)
        c = np.where(active[None, :], 10.0 ** np.clip(lc, -30, 1), 1e-30)
        T = c @ S
        ok &= (T > 0).all(1)
        keep_x.append(x[ok]); keep_c.append(c[ok]); keep_T.append(T[ok])
    return (np.concatenate(keep_T)[:n], np.concatenate(keep_x)[:n], np.concatenate(keep_c)[:n])


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
    # ---- the reference's uranium tableau (17 x 95) with known answers and the
    #      reference's PCF + Anderson on them
    Su, lku, csu, names = parse_uranium_tableau(ref_root)
    Tu, xu, cu = uranium_samples(Su, lku, 64, seed=95)
    outu, itu, cvu = o.ref_pcf_solve(Su, lku, csu, cu)
    cold = wl.cold_species(Su, Tu, csu)
    outc, itc, cvc = o.ref_pcf_solve(Su, lku, csu, cold)
    np.savez(os.path.join(HERE, "uranium_tableau.npz"), S=Su, logk=lku, comp_species=np.array(csu),
             components=np.array(names), totals=Tu, xstar=xu, cstar=cu, pcf_out=outu, pcf_it=itu, pcf_cv=cvu,
             cold=cold, pcf_cold_out=outc, pcf_cold_it=itc, pcf_cold_cv=cvc)
    print("uranium tableau %dx%d; PCF converged %d/%d from the known answers, %d/%d from the cold vectors"
          % (Su.shape[1], Su.shape[0], int(cvu.sum()), cvu.size, int(cvc.sum()), cvc.size))


if __name__ == "__main__":
    main()
