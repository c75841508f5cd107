"""FP32 emulation (numpy, CPU) of the expanded-distance evaluation used by the Gaussian FP32 kernels.

The kernels evaluate, for targets y and sources x taken relative to the centre of the target block (scaled so that
the kernel is 2^-|y-x|^2), the bracket |x|^2 - 2 y.x with three FMAs from staged -2x and |x|^2, and multiply the
target's sums by 2^-|y|^2 once; ops that sum f (y - x) write it y S - sum f x. Both identities are exact; these
tests bound the FP32 rounding they add for blocks at the radius bounds the kernels use (radius^2 64 for the
exponent, 32 for the y S - sum f x rewrite) against the float64 sums, far below the GPU tests' 2e-5 tolerance.
The exponential itself is taken exact here (the hardware ex2 adds the same error to both forms).
"""
import numpy as np

F32 = np.float32


def fma32(a, b, c):
    # a*b is exact in float64 for float32 inputs; one rounding of the sum to float32
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F32)


def ball(rng, n, r):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v * r * rng.random((n, 1)) ** (1 / 3)


def rel(u, ref):
    return np.linalg.norm(u - ref) / np.linalg.norm(ref)


def test_expanded_exponent_at_the_radius_bound():
    rng = np.random.default_rng(0)
    r2 = 64.0
    y = ball(rng, 256, np.sqrt(r2)).astype(F32)
    x = ball(rng, 2048, np.sqrt(r2) + 6).astype(F32)
    a = rng.normal(size=(2048, 3))
    d2 = ((y[:, None, :].astype(np.float64) - x[None].astype(np.float64)) ** 2).sum(-1)
    truth = np.exp2(-d2) @ a
    X = (-2 * x).astype(F32)
    q = (x.astype(np.float64) ** 2).sum(1).astype(F32)
    shape = d2.shape
    arg = fma32(np.broadcast_to(y[:, None, 2], shape), np.broadcast_to(X[None, :, 2], shape),
                np.broadcast_to(q[None], shape))
    arg = fma32(np.broadcast_to(y[:, None, 1], shape), np.broadcast_to(X[None, :, 1], shape), arg)
    arg = fma32(np.broadcast_to(y[:, None, 0], shape), np.broadcast_to(X[None, :, 0], shape), arg)
    e = np.exp2(-arg.astype(np.float64)).astype(F32)
    out = (e.astype(np.float64) @ a) * np.exp2(-(y.astype(np.float64) ** 2).sum(1))[:, None]
    assert rel(out, truth) < 2e-6


def test_centre_term_rewrite_at_the_radius_bound():
    rng = np.random.default_rng(1)
    r2 = 32.0
    y = ball(rng, 128, np.sqrt(r2)).astype(F32)
    x = ball(rng, 1024, np.sqrt(r2) + 5).astype(F32)
    w = rng.normal(size=(128, 1024))
    d = y[:, None, :].astype(np.float64) - x[None].astype(np.float64)
    f = (np.exp2(-(d ** 2).sum(-1)) * w).astype(F32)
    truth = np.einsum('kl,klc->kc', f.astype(np.float64), d)

    def tile_sums(v):  # float32 sums over tiles of 128 sources, tiles added in float64 (compensated merge)
        out = np.zeros(v.shape[0])
        for t in range(0, v.shape[1], 128):
            acc = np.zeros(v.shape[0], F32)
            for col in range(t, min(t + 128, v.shape[1])):
                acc = (acc + v[:, col]).astype(F32)
            out += acc
        return out

    S = tile_sums(f)
    E = np.stack([tile_sums((f * x[None, :, c]).astype(F32)) for c in range(3)], 1)
    out = y.astype(np.float64) * S[:, None] - E
    assert rel(out, truth) < 1e-6
