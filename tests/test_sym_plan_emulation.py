"""CPU emulation of the symmetric pair kernel's schedule (csrc/pairs_sym.cuh): the row-major units of the upper
block triangle, the stream-K split over CTAs, the row partial slots, the column partial layout and the epilogue's
reads. With a symmetric kernel matrix Kf and a payload v, the row credit of unit (i, t) is Kf[block i, tile t] v[tile]
and the column credit Kf[block i, tile t]^T v[block i]; the epilogue's sums must give Kf v for every point, every
index must stay inside its buffer, and every ordered pair must be credited exactly once."""
import numpy as np
import pytest


def row_off(i, TT, RT):
    return i * TT - RT * (i * (i - 1) // 2)


def tri(j):
    return j * (j - 1) // 2


def sk_start(c, W, C):
    return c * W // C


def sk_cta_of(u, W, C):
    c = ((u + 1) * C - 1) // W
    while c + 1 < C and sk_start(c + 1, W, C) <= u:
        c += 1
    while c > 0 and sk_start(c, W, C) > u:
        c -= 1
    return c


def plan(n, TPB, RT, wave):
    B = TPB * RT
    nblk = -(-n // B)
    TT = -(-n // TPB)
    U = row_off(nblk, TT, RT)
    C = min(U, wave)
    S = max(sk_cta_of(row_off(i + 1, TT, RT) - 1, U, C) - sk_cta_of(row_off(i, TT, RT), U, C) + 1
            for i in range(nblk))
    return nblk, TT, U, C, S


def emulate(n, TPB, RT, wave, rng):
    B = TPB * RT
    nblk, TT, U, C, S = plan(n, TPB, RT, wave)
    x = rng.normal(size=(n, 3))
    Kf = np.exp(-((x[:, None] - x[None]) ** 2).sum(-1))
    v = rng.normal(size=n)
    row_ws = np.full((S, n), np.nan)
    col_ws = np.full(tri(nblk) * B, np.nan)
    credited = np.zeros((n, n), dtype=np.int64)
    for cta in range(C):
        u, u_end = sk_start(cta, U, C), sk_start(cta + 1, U, C)
        i = max(k for k in range(nblk) if row_off(k, TT, RT) <= u) if u < u_end else 0
        while u < u_end:
            off = row_off(i, TT, RT)
            cnt = TT - RT * i
            t0, t1 = u - off, min(cnt, u_end - off)
            slot = cta - sk_cta_of(off, U, C)
            assert 0 <= slot < S
            rows = np.arange(i * B, min(i * B + B, n))
            acc = np.zeros(len(rows))
            for tt in range(t0, t1):
                t = RT * i + tt
                assert t < TT
                src = np.arange(t * TPB, min(t * TPB + TPB, n))
                acc += Kf[np.ix_(rows, src)] @ v[src]
                credited[np.ix_(rows, src)] += 1
                if tt >= RT:
                    j = t // RT
                    assert i < j < nblk
                    colsum = Kf[np.ix_(rows, src)].T @ v[rows]
                    credited[np.ix_(src, rows)] += 1
                    for r, l in enumerate(src):
                        idx = (tri(j) + i) * B + (t - RT * j) * TPB + r
                        assert 0 <= idx < col_ws.size
                        col_ws[idx] = colsum[r]
            row_ws[slot, rows] = acc
            u += t1 - t0
            i += 1
    # the epilogue (finalize_sym_kernel): tpp threads per point; thread (j, p) of a CTA of 256 threads sums slots
    # j, j + tpp, ... and column partials j, j + tpp, ... of point blockIdx * (256 / tpp) + p; thread (0, p) adds the
    # tpp sums in the order j = 0, 1, ...
    tpp = finalize_tpp(S, nblk)
    npc = 256 // tpp
    out = np.zeros(n)
    for cta in range(-(-n // npc)):
        for p in range(npc):
            idx = cta * npc + p
            if idx >= n:
                continue
            b, r = idx // B, idx % B
            nslot = (sk_cta_of(row_off(b + 1, TT, RT) - 1, U, C) - sk_cta_of(row_off(b, TT, RT), U, C) + 1)
            assert nslot <= S
            read_s, read_q, part = [], [], []
            for j in range(tpp):
                acc = 0.0
                for sl in range(j, nslot, tpp):
                    acc += row_ws[sl, idx]
                    read_s.append(sl)
                for q in range(j, b, tpp):
                    k = (tri(b) + q) * B + r
                    assert 0 <= k < col_ws.size
                    acc += col_ws[k]
                    read_q.append(q)
                part.append(acc)
            assert sorted(read_s) == list(range(nslot)) and sorted(read_q) == list(range(b))
            out[idx] = sum(part)
    return out, Kf @ v, credited


def finalize_tpp(S, nblk):
    """sym_finalize_tpp: threads per point of the epilogue (chains of about four, at most 8)."""
    t = 1
    while t < 8 and S + nblk > 4 * t:
        t *= 2
    return t


@pytest.mark.parametrize('n,TPB,RT,wave', [(1, 128, 4, 296), (100, 128, 4, 296), (511, 32, 4, 7), (513, 32, 4, 7),
                                           (2000, 32, 4, 13), (2000, 64, 2, 5), (1500, 32, 4, 1000), (777, 32, 6, 3),
                                           (2100, 128, 8, 444), (3000, 32, 8, 17)])
def test_symmetric_schedule_credits_every_pair_once(n, TPB, RT, wave):
    rng = np.random.default_rng(n + TPB + RT + wave)
    out, ref, credited = emulate(n, TPB, RT, wave, rng)
    assert np.all(credited == 1)
    assert np.allclose(out, ref, rtol=1e-12, atol=1e-12)
