"""Reference callers import the matching classes, the kernel and the surface container by the reference's module
paths (Examples/surfaceMatchingExample.py:16-20). Those imports resolve to the device classes of this package."""


def test_reference_import_paths_resolve_to_device_classes():
    from base.secondOrderSurfaceMatching import SecondOrderSurfaceMatching
    from base.surfaceMatching import SurfaceMatching
    from base.surfaces import Surface
    from base.kernelFunctions import Kernel
    from base import surfaceMatching as sm

    assert SecondOrderSurfaceMatching is sm.SecondOrderSurfaceMatching
    assert issubclass(SecondOrderSurfaceMatching, sm._DeviceMatching)
    assert issubclass(SurfaceMatching, sm._DeviceMatching)
    # the optimiser protocol the reference's bfgs drives
    for name in ('objectiveFun', 'updateTry', 'getGradient', 'acceptVarTry', 'optimizeMatching', 'resetPK'):
        assert callable(getattr(SecondOrderSurfaceMatching, name))
    assert Surface.__module__ == 'base.surfaces'
    assert Kernel.__module__ == 'base.kernelFunctions'


def test_reference_pointevolution_and_distance_names():
    from base import pointEvolution as evol
    from base import surfaceDistances as sd
    for name in ('landmarkDirectEvolutionEuler', 'landmarkHamiltonianCovector', 'landmarkHamiltonianGradient',
                 'secondOrderEvolution', 'secondOrderCovector', 'secondOrderGradient', 'landmarkEPDiff'):
        assert callable(getattr(evol, name)), name
    for name in ('varifoldNorm0', 'varifoldNormDef', 'varifoldNormGradient', 'currentNorm0', 'currentNormDef',
                 'currentNormGradient', 'measureNorm0', 'measureNormDef', 'measureNormGradient'):
        assert callable(getattr(sd, name)), name
