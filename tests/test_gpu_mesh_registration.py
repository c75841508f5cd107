"""A short registration on a real mesh (the hippocampus surface of the reference's test data), and the result
record written in the layout of the reference's saveHdf5 (as .npz)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('cls_name', ['SecondOrderSurfaceMatching', 'SurfaceMatching'])
def test_hippocampus_registration_and_result_record(cls_name, tmp_path):
    import torch
    from base import surfaceMatching as sm
    from base.kernelFunctions import Kernel
    from base.surfaces import Surface
    src = Surface(surf=os.path.join(GOLDEN, 'meshes', 'Hippo.vtk'))
    c = src.vertices.mean(axis=0)
    x1 = c + np.array([1.08, 0.95, 1.0]) * (src.vertices - c) + np.array([0.5, -0.3, 0.2])   # a mild affine change
    tgt = Surface(surf=(src.faces, x1))
    K = Kernel(name='gauss', sigma=5.0)
    K.pk_dtype = 'float32'
    opts = dict(maxIter=3, affine='none', regWeight=1.0, KparDiff=K, KparDist=('gauss', 2.0), sigmaError=1.0,
                errorType='varifold', pk_dtype='float32', algorithm='bfgs', timeStep=0.1, verb=False)
    f = getattr(sm, cls_name)(Template=src, Target=tgt, options=opts)
    obj_init = f.objectiveFun()
    f.optimizeMatching()
    torch.cuda.synchronize()
    assert len(f.history) >= 3 and np.isfinite(f.history[-1])
    assert f.history[-1] < 0.9 * obj_init        # three BFGS steps make real progress
    path = f.saveHdf5(os.path.join(tmp_path, 'output.h5'))
    assert path.endswith('output.npz')
    d = np.load(path)
    g = 'LDDMM Results/'
    for k in ('parameters/Time steps', 'parameters/Deformation Kernel type', 'parameters/Deformation Kernel width',
              'parameters/Spatial Varifold width', 'template/vertices', 'template/faces', 'target/vertices',
              'target/faces', 'deformedTemplate/vertices', 'variables/alpha', 'variables/affine',
              'descriptors/Jacobian', 'descriptors/Surface Jacobian', 'descriptors/Displacement'):
        assert g + k in d.files, k
    nv = src.vertices.shape[0]
    assert int(d[g + 'parameters/Time steps']) == 10
    assert d[g + 'deformedTemplate/vertices'].shape == (nv, 3)
    assert d[g + 'descriptors/Jacobian'].shape == (nv, 1)
    assert np.allclose(d[g + 'descriptors/Displacement'], d[g + 'deformedTemplate/vertices'] - src.vertices)
    sj = d[g + 'descriptors/Surface Jacobian']
    assert sj.shape == (nv,) and np.all(sj > 0)
