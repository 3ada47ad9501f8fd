"""The permutation pass (run_perm_pass in qk_pass_device.cuh) computes, per
thread, the state offset of tile element f = tid + i NT and the shared-memory
indices of f and of perm(f) as the thread's part combined with the parts of
the set bits of i (OR for the offset, XOR for the swizzled index).  That is
exact because the bit deposit (pass_off), the bit-pair swaps (perm_bits) and
the swizzle (swz) are each linear over disjoint bits.  Restated here in
Python for random tile shapes (both amplitude types, up to 14 tile bits, up
to 512 threads a tile): the decomposed values equal the direct ones, the
shared-memory indices stay in the tile, and the pass leaves element j at the
position of perm(j)."""
import random


def pass_off(j, T, L, bpos):
    g = j & ((1 << L) - 1)
    for k in range(L, T):
        g |= ((j >> k) & 1) << bpos[k]
    return g


def perm_bits(j, pa, pb):
    f = j
    for a, b in zip(pa, pb):
        x, y = (j >> a) & 1, (j >> b) & 1
        f = (f & ~(1 << a) & ~(1 << b)) | (y << a) | (x << b)
    return f


def swz(j, c128):
    if c128:
        return j ^ (((j >> 3) ^ (j >> 6) ^ (j >> 9) ^ (j >> 12)) & 7)
    return j ^ (((j >> 4) ^ (j >> 8) ^ (j >> 12)) & 15)


def test_thread_offsets_match_direct_values():
    rng = random.Random(7)
    for _ in range(60):
        n = rng.randint(6, 34)
        c128 = rng.random() < 0.5
        T = rng.randint(2, min(n, 13 if c128 else 14))
        bpos = sorted(rng.sample(range(n), T))
        L = 0
        while L < T and bpos[L] == L:
            L += 1
        k = rng.randint(1, min(6, T // 2))
        bits = rng.sample(range(T), 2 * k)
        pa, pb = bits[:k], bits[k:]
        N = 1 << T
        NT = min(512, N)
        parts = [NT << b for b in range(5) if (NT << b) < N]
        assert 1 << len(parts) == N // NT
        g_u = [pass_off(m, T, L, bpos) for m in parts]
        sw_u = [swz(m, c128) for m in parts]
        sp_u = [swz(perm_bits(m, pa, pb), c128) for m in parts]
        buf = [None] * N
        pos = {}
        for tid in range(NT):
            g_t, sw_t, sp_t = pass_off(tid, T, L, bpos), swz(tid, c128), swz(perm_bits(tid, pa, pb), c128)
            for i in range(N // NT):
                a, x, y = g_t, sw_t, sp_t
                for b in range(len(parts)):
                    if (i >> b) & 1:
                        a, x, y = a | g_u[b], x ^ sw_u[b], y ^ sp_u[b]
                f = tid + i * NT
                assert a == pass_off(f, T, L, bpos)
                assert x == swz(f, c128) and y == swz(perm_bits(f, pa, pb), c128)
                assert 0 <= x < N and 0 <= y < N and buf[x] is None
                buf[x] = f            # load: element f (at pass_off(f)) into the tile
                pos[a] = y            # store: position pass_off(f) takes the tile's entry y
        out = {a: buf[y] for a, y in pos.items()}
        assert len(out) == N
        for j in range(N):
            assert out[pass_off(perm_bits(j, pa, pb), T, L, bpos)] == j
