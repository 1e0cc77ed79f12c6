"""Volume file conversion and cropping (the reference's src/cutFile.cu).

    python -m visualtur_b200.convert IN OUT [--dataset value] [--out-dataset value]
                                     [--format hdf5|raw] [--crop X,Y,Z,DIM | --box X0,Y0,Z0,X1,Y1,Z1]

Without a crop, the whole dataset is rewritten in the other container
(raw VTVOL001 <-> HDF5) with its voxel type kept.  With --crop, as cutFile
does, the cube [X, X+DIM) x [Y, Y+DIM) x [Z, Z+DIM) is read with
FileManager::readHDF5_Voxel_Array semantics (float32, zero outside the
volume) and written as a float32 dataset; --box takes any box [X0, X1) x
[Y0, Y1) x [Z0, Z1).
"""
import argparse

import numpy as np


def convert(src, dst, dataset="value", out_dataset="value", fmt="hdf5", box=None):
    """Writes `dst` from the dataset of `src`; box = ((x0,y0,z0), (x1,y1,z1))
    crops as cutFile does.  Returns the written array's shape and dtype."""
    import visualtur_b200 as vt
    fm = vt.FileManager(src, dataset)
    try:
        if box is None:
            data = fm.readHDF5()
        else:
            s, e = box
            data = fm.readHDF5_Voxel_Array(s, e)
    finally:
        fm.close()
    vt.FileManager.CreateFile(data, dst, out_dataset, fmt=1 if fmt == "hdf5" else 0)
    return data.shape, data.dtype


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("src")
    ap.add_argument("dst")
    ap.add_argument("--dataset", default="value")
    ap.add_argument("--out-dataset", default="value")
    ap.add_argument("--format", choices=("hdf5", "raw"), default="hdf5")
    g = ap.add_mutually_exclusive_group()
    g.add_argument("--crop", help="X,Y,Z,DIM (cutFile)")
    g.add_argument("--box", help="X0,Y0,Z0,X1,Y1,Z1")
    a = ap.parse_args(argv)
    box = None
    if a.crop:
        x, y, z, d = (int(v) for v in a.crop.split(","))
        box = ((x, y, z), (x + d, y + d, z + d))
    elif a.box:
        v = [int(t) for t in a.box.split(",")]
        box = (tuple(v[:3]), tuple(v[3:]))
    shape, dtype = convert(a.src, a.dst, a.dataset, a.out_dataset, a.format, box)
    print("%s: %s %s" % (a.dst, "x".join(str(n) for n in shape), np.dtype(dtype).name))


if __name__ == "__main__":
    main()
