"""Copy the reference's example inputs that the host driver runs into this
folder, so that the GPU tests can run them where the reference tree is absent.

    python tests/golden/examples/make_examples.py [REFERENCE_ROOT]

For each supported example (examples/<name>/ of the reference: CompLaB.xml and
input/*) the files are copied unchanged into tests/golden/examples/<name>/.
The reference keeps each example's rate law in a compiled header
(examples/<name>/defineKinetics.hh, defineAbioticKinetics.hh); the table form
of those laws, which the driver reads with --rates, is the hand-written
rates.xml beside each copy (not produced by this script).  Example 11's
network, which the reference compiles in from surrogateModel.hh, is written
here as shipped_network.txt (the driver's --surrogate file) from the golden
fixture surrogate_shipped.npz.  The header and the
table are compared on random inputs by
tests/test_oracle_pins.py::test_oracle_rates_match_example_headers and
tests/test_ratelaw_port.py.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE))))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "tests"))

SUPPORTED = ["01_flow_only", "02_diffusion_only", "03_abiotic_kinetics", "04_equilibrium",
             "05_biotic_cellular_automaton", "06_biotic_finite_difference", "07_biotic_lattice_boltzmann",
             "08_two_microbes", "11_surrogate",
             "13_precipitation", "14_dissolution", "15_precip_and_dissolution"]


def write_network(npz_path, out_path):
    """The shipped surrogate network (tests/golden/surrogate_shipped.npz, made
    from the reference's surrogateModel.hh by make_golden.py) as the host
    driver's network file (--surrogate)."""
    import numpy as np
    z = np.load(npz_path)
    L = sum(1 for k in z.files if k.startswith("W"))
    W = [z["W%d" % l] for l in range(L)]
    widths = [W[0].shape[1]] + [w.shape[0] for w in W]
    f = lambda a: " ".join(repr(float(v)) for v in np.ravel(a))
    lines = ["# the surrogate network the reference compiles in (surrogateModel.hh)",
             "layers %d" % L, "widths " + " ".join(str(w) for w in widths)]
    for l in range(L):
        lines += ["W%d %s" % (l, f(W[l])), "b%d %s" % (l, f(z["b%d" % l]))]
    lines += ["x_offset " + f(z["x_offset"]), "x_gain " + f(z["x_gain"]), "x_ymin " + f(z["x_ymin"]),
              "y_offset " + f(z["y_offset"]), "y_gain " + f(z["y_gain"]), "y_ymin " + f(z["y_ymin"])]
    open(out_path, "w").write("\n".join(lines) + "\n")


def main():
    from conftest import reference_root
    root = sys.argv[1] if len(sys.argv) > 1 else reference_root()
    if not root:
        raise SystemExit("no reference tree: pass its path or set COMPLAB_REFERENCE")
    for name in SUPPORTED:
        src = os.path.join(root, "examples", name)
        dst = os.path.join(HERE, name)
        os.makedirs(os.path.join(dst, "input"), exist_ok=True)
        shutil.copyfile(os.path.join(src, "CompLaB.xml"), os.path.join(dst, "CompLaB.xml"))
        for f in sorted(os.listdir(os.path.join(src, "input"))):
            shutil.copyfile(os.path.join(src, "input", f), os.path.join(dst, "input", f))
        if name == "11_surrogate":
            write_network(os.path.join(os.path.dirname(HERE), "surrogate_shipped.npz"),
                          os.path.join(dst, "shipped_network.txt"))
        print("copied", name)


if __name__ == "__main__":
    main()
