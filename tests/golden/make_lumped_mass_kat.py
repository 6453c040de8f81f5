"""Builds tests/golden/lumped_mass_kat.npz from the reference's own example.

The reference ships one known-answer vector for the explicit path:
examples/02_explicit_fluid_VMS/06_2D_hexa_lid_driven_cavity/lumped_mass.txt,
the row-sum lumped mass l_M[node*3+c] that
femSUPGExplicitFluidSolver.cpp:507-598 (form_lumped_mass) produced with
rho = 10 (VMSPROPS 10.0 ..., create_exVMS_simul.py) on the 99x99x1 hexa8 mesh
stored in fluid.vtu of the same folder.

This script decodes fluid.vtu (appended base64, zlib blocks, UInt32 headers),
cuts a block of elements out of the mesh and keeps the lumped-mass values of
the nodes whose every incident element lies in that block (those values are
complete within the block).  The resulting fixture is a few tens of KB.

Run from the repository root:  python tests/golden/make_lumped_mass_kat.py [reference_root]
(default: $FEMORPH_REFERENCE, else /root/reference)
"""
import base64
import os
import re
import sys
import zlib

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FEMORPH_REFERENCE", "/root/reference")
EX = os.path.join(REF, "examples/02_explicit_fluid_VMS/06_2D_hexa_lid_driven_cavity")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lumped_mass_kat.npz")


def read_vtu(path):
    txt = open(path, "rb").read()
    head, app = txt.split(b'<AppendedData encoding="base64">', 1)
    raw = app.split(b"_", 1)[1].split(b"</AppendedData>")[0].strip()
    arrays = {}
    for m in re.finditer(rb'<DataArray type="(\w+)"[^>]*Name="(\w+)"[^>]*offset="(\d+)"', head):
        arrays[m.group(2).decode()] = (m.group(1).decode(), int(m.group(3)))
    dt = {"Float64": np.float64, "Int64": np.int64, "Int32": np.int32, "UInt8": np.uint8}

    def decode(name):
        typ, off = arrays[name]
        # header: nblocks, blocksize, lastblocksize, compressed sizes (UInt32)
        h0 = base64.b64decode(raw[off:off + 8])  # first 4 bytes are enough
        nb = int(np.frombuffer(base64.b64decode(raw[off:off + 24])[:4], np.uint32)[0])
        hlen = 4 * (3 + nb)
        henc = 4 * ((hlen + 2) // 3)
        hdr = np.frombuffer(base64.b64decode(raw[off:off + henc])[:hlen], np.uint32)
        csz = hdr[3:3 + nb]
        denc = 4 * ((int(csz.sum()) + 2) // 3)
        data = base64.b64decode(raw[off + henc:off + henc + denc])
        out, p = [], 0
        for s in csz:
            out.append(zlib.decompress(data[p:p + int(s)]))
            p += int(s)
        return np.frombuffer(b"".join(out), dt[typ])

    return decode


def main():
    dec = read_vtu(os.path.join(EX, "fluid.vtu"))
    pts = dec("Points").reshape(-1, 3)
    conn = dec("connectivity").reshape(-1, 8).astype(np.int64)
    lm = np.loadtxt(os.path.join(EX, "lumped_mass.txt"))
    assert lm.size == pts.shape[0] * 3
    # element block: centroids in [0.3, 0.5] x [0.3, 0.5]
    cen = pts[conn].mean(axis=1)
    sel = np.nonzero((cen[:, 0] > 0.3) & (cen[:, 0] < 0.5) & (cen[:, 1] > 0.3) & (cen[:, 1] < 0.5))[0]
    sub = conn[sel]
    nodes, inv = np.unique(sub, return_inverse=True)
    count_all = np.bincount(conn.ravel(), minlength=pts.shape[0])
    count_sub = np.bincount(sub.ravel(), minlength=pts.shape[0])
    complete = nodes[count_sub[nodes] == count_all[nodes]]
    local = np.searchsorted(nodes, complete)
    np.savez_compressed(OUT, coords=pts[nodes], conn=inv.reshape(-1, 8).astype(np.int32),
                        rho=np.float64(10.0), check_nodes=local.astype(np.int32),
                        lumped_mass=lm.reshape(-1, 3)[complete])
    print(f"wrote {OUT}: {sel.size} elements, {nodes.size} nodes, {complete.size} checked")


if __name__ == "__main__":
    main()
