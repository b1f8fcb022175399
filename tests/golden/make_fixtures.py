"""Regenerates the committed fixtures under tests/golden/ (run in a container
that has the reference checkout and the oracle built with `make -C oracle ref`):

  data/cc-pvdz/cc-pvdz.gbs        cc-pVDZ blocks for H, C, N, O, cut from the
  data/cc-pVDZ-RI/cc-pVDZ-RI.gbs  reference's data/ files (element blocks verbatim)
  data/cc-pvdz/{H,C,N,O}.dat      the reference's SAD guesses for those elements
  data/water.xyz, data/c10h22.xyz, data/c20h42.xyz, data/c40h82.xyz
                                  synthetic geometries (yatscf-df_b200/geometry.py)
  water_ref.npz, c10h22_ref.npz   outputs of the reference's own SCF code
                                  (oracle/_ref/ref_dump) on those inputs
  c20h42_ref.npz, c40h82_ref.npz  the same for the two large alkanes, kept
                                  small: the energy trajectory to |dE| < 1e-11,
                                  the screening mask as packed bits, and every
                                  RSTEP-th row of the iteration-0 J, K and of
                                  the guess factor Cocc

The reference checkout is taken from the first argument, else from the
environment variable TINYSCF_REFERENCE, else from BASELINE.json's
reference_path. With --dumps DIR the ref_dump outputs are kept in (or, when
present, read back from) DIR/<name>; --only limits the run to some molecules.

Usage: python tests/golden/make_fixtures.py [/path/to/reference] [--dumps DIR] [--only name,name]
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "yatscf-df_b200"))
import geometry  # noqa: E402

ELEMENTS = ["H", "C", "N", "O"]


def cut_gbs(src, dst, elements):
    """Keep the header line and the blocks of the listed elements."""
    with open(src) as f:
        lines = f.read().splitlines(keepends=True)
    out = [lines[0], "****\n"]
    i = 1
    while i < len(lines):
        tok = lines[i].split()
        if lines[i][:1].isalpha() and tok and tok[0] in elements:
            j = i
            while j < len(lines) and not lines[j].startswith("****"):
                j += 1
            out.extend(lines[i:j + 1])
            i = j + 1
        else:
            i += 1
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    with open(dst, "w") as f:
        f.writelines(out)


def read_dump(d, nbf, nocc, naux, iters=(0, 1, 2), keep_B=False):
    def ld(name, shape, dt=np.float64):
        return np.fromfile(os.path.join(d, name), dtype=dt).reshape(shape)
    out = {}
    for name in ("S", "H", "X", "D0"):
        out[name] = ld(name + ".bin", (nbf, nbf))
    out["Cocc0"] = ld("Cocc0.bin", (nbf, nocc))
    out["mask"] = ld("mask.i32", (nbf, nbf), np.int32)
    for k in iters:
        for name in ("J", "K", "F", "Fo", "D"):
            out["it%d_%s" % (k, name)] = ld("it%d_%s.bin" % (k, name), (nbf, nbf))
        out["it%d_Cocc" % k] = ld("it%d_Cocc.bin" % k, (nbf, nocc))
    e = np.loadtxt(os.path.join(d, "energies.txt"))
    out["energies"] = e[:, 1]
    out["hf_energies"] = e[:, 2]
    if keep_B:
        nnz = int(out["mask"].max()) + 1
        out["B"] = ld("B.bin", (nnz, naux))
    return out


def run_ref(ref_dump, bas, dfbas, xyz, niters, outdir, dumpB):
    subprocess.run([ref_dump, bas, dfbas, xyz, str(niters), outdir, "1" if dumpB else "0"],
                   check=True, stdout=subprocess.DEVNULL)
    meta = dict(l.split() for l in open(os.path.join(outdir, "meta.txt")))
    return {k: (float(v) if "." in v or "e" in v else int(v)) for k, v in meta.items()}


# Row stride of the iteration-0 J/K rows kept for the large molecules.
RSTEP = {"c20h42": 3, "c40h82": 8}


def compact_large(d, meta):
    """Fixture of a large molecule: energies, packed mask, sampled J/K rows."""
    nbf = meta["nbf"]

    def ld(name, shape, dt=np.float64):
        return np.fromfile(os.path.join(d, name), dtype=dt).reshape(shape)
    e = np.loadtxt(os.path.join(d, "energies.txt"))
    mask = ld("mask.i32", (nbf, nbf), np.int32)
    rows = np.arange(0, nbf, RSTEP[meta["name"]])
    return {
        "energies": e[:, 1], "hf_energies": e[:, 2],
        "mask_bits": np.packbits((mask >= 0).ravel()), "nbf": np.array(nbf), "nnz": np.array(meta["nnz"]),
        "rows": rows, "it0_J_rows": ld("it0_J.bin", (nbf, nbf))[rows], "it0_K_rows": ld("it0_K.bin", (nbf, nbf))[rows],
        "Cocc0_rows": ld("Cocc0.bin", (nbf, meta["nocc"]))[rows],
    }


def reference_path(argv):
    if argv:
        return argv[0]
    if os.environ.get("TINYSCF_REFERENCE"):
        return os.environ["TINYSCF_REFERENCE"]
    with open(os.path.join(REPO, "BASELINE.json")) as f:
        return json.load(f)["reference_path"]


def main(ref, dumps=None, only=None):
    data = os.path.join(HERE, "data")
    cut_gbs(os.path.join(ref, "data/cc-pvdz/cc-pvdz.gbs"), os.path.join(data, "cc-pvdz/cc-pvdz.gbs"), ELEMENTS)
    cut_gbs(os.path.join(ref, "data/cc-pVDZ-RI/cc-pVDZ-RI.gbs"), os.path.join(data, "cc-pVDZ-RI/cc-pVDZ-RI.gbs"),
            ELEMENTS)
    for el in ELEMENTS:
        shutil.copyfile(os.path.join(ref, "data/cc-pvdz", el + ".dat"), os.path.join(data, "cc-pvdz", el + ".dat"))
    geometry.write_xyz(os.path.join(data, "water.xyz"), geometry.water())
    for n in (10, 20, 40):
        geometry.write_xyz(os.path.join(data, "c%dh%d.xyz" % (n, 2 * n + 2)), geometry.alkane(n))
    ref_dump = os.path.join(REPO, "oracle", "_ref", "ref_dump")
    bas = os.path.join(data, "cc-pvdz/cc-pvdz.gbs")
    dfbas = os.path.join(data, "cc-pVDZ-RI/cc-pVDZ-RI.gbs")
    for name, niters in (("c20h42", 30), ("c40h82", 30)):
        if only and name not in only:
            continue
        d = os.path.join(dumps, name) if dumps else tempfile.mkdtemp()
        if not os.path.exists(os.path.join(d, "meta.txt")):
            os.makedirs(d, exist_ok=True)
            run_ref(ref_dump, bas, dfbas, os.path.join(data, name + ".xyz"), niters, d, False)
        meta = dict(l.split() for l in open(os.path.join(d, "meta.txt")))
        meta = {k: (float(v) if "." in v or "e" in v else int(v)) for k, v in meta.items()}
        meta["name"] = name
        fx = compact_large(d, meta)
        fx["nuc_energy"] = np.array(meta["nuc_energy"])
        np.savez_compressed(os.path.join(HERE, name + "_ref.npz"), **fx)
        print(name, meta, "E =", fx["energies"][-1])
        if not dumps:
            shutil.rmtree(d)
    for name, niters, dumpB in (("water", 30, True), ("c10h22", 30, False)):
        if only and name not in only:
            continue
        with tempfile.TemporaryDirectory() as td:
            meta = run_ref(ref_dump, bas, dfbas, os.path.join(data, name + ".xyz"), niters, td, dumpB)
            fx = read_dump(td, meta["nbf"], meta["nocc"], meta["naux"], keep_B=dumpB)
            if name != "water":
                # keep the larger case small: energies, mask and the iteration-0/1 matrices only
                fx = {k: v for k, v in fx.items() if k in ("energies", "hf_energies", "mask", "D0", "Cocc0",
                                                           "it0_J", "it0_K", "it1_J", "it1_K", "it1_F")}
                for k in list(fx):
                    if fx[k].dtype == np.float64 and fx[k].ndim == 2:
                        fx[k] = fx[k].astype(np.float64)
            fx["nuc_energy"] = np.array(meta["nuc_energy"])
            np.savez_compressed(os.path.join(HERE, name + "_ref.npz"), **fx)
            print(name, meta, "E =", fx["energies"][-1])


if __name__ == "__main__":
    args = sys.argv[1:]
    opts = {}
    for flag in ("--dumps", "--only"):
        if flag in args:
            i = args.index(flag)
            opts[flag] = args[i + 1]
            del args[i:i + 2]
    only = opts["--only"].split(",") if "--only" in opts else None
    main(reference_path(args), opts.get("--dumps"), only)
