"""Copy the two real meshes of the reference's test data used by tests/test_mesh_io.py into tests/golden/meshes/.

    python tests/golden/make_mesh_fixtures.py --ref <the reference's py-lddmm directory>

Hippo.vtk (legacy ASCII VTK polydata, 1,001 points, 1,998 triangles, a per-point scalar field) and
spot_triangulated_reduced.obj (Wavefront OBJ, triangles only) from the reference's TestData folder. They are data,
copied byte for byte; the tests need no access to the reference tree.
"""
import argparse
import os
import shutil

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = (('TestData/Hippo.vtk', 'Hippo.vtk'),
         ('TestData/Surfaces/KCrane/spot_triangulated_reduced.obj', 'spot_triangulated_reduced.obj'))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', required=True, help="the reference's py-lddmm directory")
    args = ap.parse_args()
    out = os.path.join(HERE, 'meshes')
    os.makedirs(out, exist_ok=True)
    for src, dst in FILES:
        shutil.copyfile(os.path.join(args.ref, src), os.path.join(out, dst))
        print('copied', dst)


if __name__ == '__main__':
    main()
