"""Extract the reference's own known answers for this path into lam_pins.npz.

Run once in a checkout that has the reference tree, whose root is given on
the command line or in the environment variable POLYSTRING_REFERENCE:

    python tests/golden/make_golden.py <reference root>

The output is committed so that the tests need no access to the reference at
run time.

What is taken, all from polyorder-master.zip:example/AB/LAM/ (the upstream
PolyOrder snapshot bundled in the reference):

* 1D/field_in_64.mat, 2D/field_in_32x32.mat: the input fields wA, wB used by
  those example runs (Grid gridInitType = File).
* {1D,2D}/param.ini: the example config files, copied unchanged to
  lam1d_param.ini and lam2d_param.ini.
* string/paramString.ini and an excerpt of string/defect.mat (string_files
  below), for the string application's tests.
* {1D,2D}/cell_opt_{rqm4,rqm4_anderson,os2,os2_anderson}.mat and
  1D/cell_opt_{etdrk4,etdrk4_anderson}.mat: the (a, F)
  pairs written by scft::save_cell (src/scft.cc:589-609) during the Brent
  cell optimisation.  Every entry is a converged SCFT free energy H at cell
  size a (1D: thresh_residual 1e-8; 2D: 1e-6), with Ms = [51, 51],
  chiN = 30, f = 0.5, incompressible, Simpson contour integration,
  lam = [0.05, 0.05, 5.0], n_Anderson_mixing = 5 (the param.ini files).
"""
import io
import os
import struct
import sys
import zipfile

import numpy as np
import scipy.io


def main(ref_root):
    z = zipfile.ZipFile(os.path.join(ref_root, "polyorder-master.zip"))
    base = "polyorder-master/example/AB/LAM/"
    out = {}
    f1 = scipy.io.loadmat(io.BytesIO(z.read(base + "1D/field_in_64.mat")))
    out["lam1d_wA"] = np.asarray(f1["wA"], dtype=np.float64).reshape(64, 1, 1)
    out["lam1d_wB"] = np.asarray(f1["wB"], dtype=np.float64).reshape(64, 1, 1)
    f2 = scipy.io.loadmat(io.BytesIO(z.read(base + "2D/field_in_32x32.mat")))
    out["lam2d_wA"] = np.asarray(f2["wA"], dtype=np.float64).reshape(32, 32, 1)
    out["lam2d_wB"] = np.asarray(f2["wB"], dtype=np.float64).reshape(32, 32, 1)
    for dim in ("1D", "2D"):
        for tag in ("rqm4", "rqm4_anderson", "os2", "os2_anderson"):
            name = base + "%s/cell_opt_%s.mat" % (dim, tag)
            d = scipy.io.loadmat(io.BytesIO(z.read(name)))
            key = "%s_%s" % (dim.lower(), tag)
            out[key + "_a"] = np.asarray(d["a"], dtype=np.float64).ravel()
            out[key + "_F"] = np.asarray(d["F"], dtype=np.float64).ravel()
    for tag in ("etdrk4", "etdrk4_anderson"):   # ETDRK4 traces exist for 1D only
        d = scipy.io.loadmat(io.BytesIO(z.read(base + "1D/cell_opt_%s.mat" % tag)))
        out["1d_%s_a" % tag] = np.asarray(d["a"], dtype=np.float64).ravel()
        out["1d_%s_F" % tag] = np.asarray(d["F"], dtype=np.float64).ravel()
    here = os.path.dirname(os.path.abspath(__file__))
    # the example config files themselves, unchanged (inputs of the driver test)
    for dim in ("1D", "2D"):
        with open(os.path.join(here, "lam%s_param.ini" % dim.lower()), "wb") as f:
            f.write(z.read(base + "%s/param.ini" % dim))
    string_files(ref_root, here)
    dst = os.path.join(here, "lam_pins.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, sorted(out))


def mat_elements(raw):
    """(offset, length, name) of the top-level data elements of a MAT-v5 file."""
    out = []
    off = 128
    while off + 8 <= len(raw):
        t, n = struct.unpack("<II", raw[off:off + 8])
        total = 8 if t >> 16 else 8 + (n + 7) // 8 * 8
        name = None
        if t == 14:                     # miMATRIX: flags, dims, then the name
            p = off + 8 + 16
            dn = struct.unpack("<I", raw[p + 4:p + 8])[0]
            p += 8 + (dn + 7) // 8 * 8
            w0 = struct.unpack("<I", raw[p:p + 4])[0]
            if w0 >> 16:
                name = raw[p + 4:p + 4 + (w0 >> 16)].decode()
            else:
                nn = struct.unpack("<I", raw[p + 4:p + 8])[0]
                name = raw[p + 8:p + 8 + nn].decode()
        out.append((off, total, name))
        off += total
    return out


def string_files(ref_root, here):
    """The string application's config, unchanged (string/paramString.ini ->
    paramString.ini), and an excerpt of its end-state file string/defect.mat:
    its 128-byte header followed, byte for byte, by the data elements of the
    variables Q, z, t and incomp.  Those are the variables whose storage the
    reader must convert: MATLAB wrote the double arrays z and incomp as
    miUINT8 and t as miUINT16 (the 128 x 352 fields are plain miDOUBLE)."""
    with open(os.path.join(ref_root, "string", "paramString.ini"), "rb") as f:
        cfg = f.read()
    with open(os.path.join(here, "paramString.ini"), "wb") as f:
        f.write(cfg)
    with open(os.path.join(ref_root, "string", "defect.mat"), "rb") as f:
        raw = f.read()
    keep = {"Q", "z", "t", "incomp"}
    parts = [raw[:128]] + [raw[o:o + n] for o, n, name in mat_elements(raw) if name in keep]
    with open(os.path.join(here, "defect_excerpt.mat"), "wb") as f:
        f.write(b"".join(parts))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("POLYSTRING_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py <reference root>  (or set POLYSTRING_REFERENCE)")
    main(root)
