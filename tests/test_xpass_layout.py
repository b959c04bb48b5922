"""The warp-per-row x pass's index arithmetic, restated lane by lane in numpy (CPU).

k_xpass_w (csrc/sns_kernels.cu) gives each warp R = 512 / N rows and runs every stage of them
in registers and through two XOR-swizzled shared-memory buffers.  This file restates, for
N = 128, 256 and 512, what each lane loads, transforms and stores in each stage -- the
packing of the staged half rows, the stage-A output swizzle (16 t + (k ^ key)), the stage-B
reads with the four-step twiddles, the split-in-frequency radix-32 combine at N = 512, the
product slots (pslot), the partner lane of the r2c unpack and the halved forward twiddles --
and checks:
  * the result equals a direct numpy FFT of the same packing (the 12 product half spectra,
    and in the diagnostic mode each row's sum of |u|^2 / 2 and max |u|^2);
  * no two lanes write the same shared-memory element, and every element is written;
  * every shared-memory access of a half-warp hits 16 distinct 8-byte bank pairs (no bank
    conflicts), for the stage-A writes, the product writes and the stage-B reads.
The GPU parity tests check the kernel itself; this pins the layout the kernel is built on.
"""
import numpy as np
import pytest


def dft(v, d):
    n = len(v)
    q = np.arange(n)
    return np.exp(d * 2j * np.pi * np.outer(q, q) / n) @ v


def w32(q):
    return np.exp(-2j * np.pi * q / 32)


class Layout:
    def __init__(self, N):
        self.N, self.M, self.R, self.NH = N, N // 16, 512 // N, N // 2
        self.S2 = 2 if N == 512 else 1
        self.MP = 2 if N == 128 else 1
        self.NZ = 16 // self.MP
        M = self.M
        tw2 = np.array([np.exp(-2j * np.pi * rr * j / N) for rr in range(M) for j in range(16)])
        self.twt = np.zeros((16, 32), complex)
        for i in range(16):
            for L in range(32):
                rr = self.S2 * i + ((L >> 4) if N == 512 else 0)
                self.twt[i, L] = tw2[rr * 16 + (L & 15)] if rr < M else 0

    def wkey(self, t, r):
        return ((t + 8 * (r & 1)) & 15) if self.N == 128 else (t & 15)

    def pslot(self, jr, k1, r):
        if self.N == 128:
            jj = jr ^ (r & 1)
            return 8 * jj + (k1 ^ ((jj >> 1) & 7))
        return self.M * jr + (k1 ^ jr)

    def row_b(self, lane, p):
        N = self.N
        return 0 if N == 512 else ((lane >> 4) if N == 256 else 2 * p + (lane >> 4))


def pack(U, V, x, N):
    """Z(x) of the staged half rows: the x-mirror and the real-part rule at 0 and N/2."""
    NH = N // 2
    if x == 0:
        return U[0].real + 1j * V[0].real
    if x < NH:
        return (U[x].real - V[x].imag) + 1j * (U[x].imag + V[x].real)
    if x == NH:
        return U[NH].real + 1j * V[NH].real
    a, b = U[N - x], V[N - x]
    return (a.real + b.imag) + 1j * (b.real - a.imag)


def assert_banks(addrs_by_half):
    for addrs in addrs_by_half.values():
        assert len({a % 16 for a in addrs}) == 16, "bank conflict"


def inverse_stages(lay, U, V, nc):
    """Stage A (with its write swizzle) and stage B; returns z[(lane, p, c)] (NZ values)."""
    N, M, R = lay.N, lay.M, lay.R
    Wc = np.full((R, 3, N), np.nan, complex)
    for c in range(nc):
        for q in range(16):
            halves = {}
            for lane in range(32):
                t, r = lane % M, lane // M
                halves.setdefault(lane >> 4, []).append((r * 3 + c) * N + 16 * t + (q ^ lay.wkey(t, r)))
            assert_banks(halves)
    for lane in range(32):
        t, r = lane % M, lane // M
        for c in range(nc):
            v = dft(np.array([pack(U[r, c], V[r, c], t + M * q, N) for q in range(16)]), +1)
            for q in range(16):
                a = 16 * t + (q ^ lay.wkey(t, r))
                assert np.isnan(Wc[r, c, a]), "two lanes write one element"
                Wc[r, c, a] = v[q]
    assert not np.isnan(Wc[:, :nc]).any()
    z = {}
    for p in range(lay.MP):
        for c in range(nc):
            for i in range(lay.NZ):
                halves = {}
                for lane in range(32):
                    j, hh = lane & 15, ((lane >> 4) if N == 512 else 0)
                    rB, rr = lay.row_b(lane, p), lay.S2 * i + hh
                    halves.setdefault(lane >> 4, []).append((rB * 3 + c) * N + 16 * rr + (j ^ lay.wkey(rr, rB)))
                assert_banks(halves)
    for lane in range(32):
        j, hh = lane & 15, ((lane >> 4) if N == 512 else 0)
        for p in range(lay.MP):
            rB = lay.row_b(lane, p)
            for c in range(nc):
                v = np.array([Wc[rB, c, 16 * (lay.S2 * i + hh) + (j ^ lay.wkey(lay.S2 * i + hh, rB))]
                              * np.conj(lay.twt[i, lane]) for i in range(lay.NZ)])
                v = dft(v, +1)
                if N == 512 and hh:
                    v = v * np.conj(w32(np.arange(16)))
                z[(lane, p, c)] = v
    if N == 512:  # radix-32 combine across the half-warps: h = 0 keeps E + T, h = 1 E - T
        z = {(lane, p, c): (z[(lane ^ 16, p, c)] - v) if lane >> 4 else (v + z[(lane ^ 16, p, c)])
             for (lane, p, c), v in z.items()}
    return z


def products_stage(lay, U, V):
    N, M, R, NH = lay.N, lay.M, lay.R, lay.NH
    z = inverse_stages(lay, U, V, 3)
    twh = lay.twt / 2
    pairs = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    P = np.full((2, 3, R, N), np.nan, complex)
    for half in range(2):
        pv = {(lane, p, ab): (lambda a, b: a.real * b.real + 1j * a.imag * b.imag)(
            z[(lane, p, pairs[ab][0])], z[(lane, p, pairs[ab][1])])
            for lane in range(32) for p in range(lay.MP) for ab in range(3 * half, 3 * half + 3)}
        for lane in range(32):
            j, hh = lane & 15, ((lane >> 4) if N == 512 else 0)
            for p in range(lay.MP):
                rB = lay.row_b(lane, p)
                for ab in range(3 * half, 3 * half + 3):
                    v = pv[(lane, p, ab)].copy()
                    if N == 512:  # split in frequency over n and n + 16
                        o = pv[(lane ^ 16, p, ab)]
                        v = (o - v) * w32(np.arange(16)) if hh else v + o
                    v = dft(v, -1)
                    for m in range(lay.NZ):
                        sl = lay.pslot(j, lay.S2 * m + hh, rB)
                        assert np.isnan(P[half, ab % 3, rB, sl]), "two lanes write one product slot"
                        P[half, ab % 3, rB, sl] = v[m] * twh[m, lane]
        for p in range(lay.MP):
            for m in range(lay.NZ):
                halves = {}
                for lane in range(32):
                    j, hh = lane & 15, ((lane >> 4) if N == 512 else 0)
                    rB = lay.row_b(lane, p)
                    halves.setdefault(lane >> 4, []).append(rB * N + lay.pslot(j, lay.S2 * m + hh, rB))
                assert_banks(halves)
        for jj in range(16):
            halves = {}
            for lane in range(32):
                k1, r = lane % M, lane // M
                halves.setdefault(lane >> 4, []).append(r * N + lay.pslot(jj, k1, r))
            assert_banks(halves)
    assert not np.isnan(P).any()
    out = np.zeros((R, 12, NH + 1), complex)
    X = {(lane, ab): dft(np.array([P[ab // 3, ab % 3, lane // M, lay.pslot(jj, lane % M, lane // M)]
                                   for jj in range(16)]), -1) for lane in range(32) for ab in range(6)}
    for lane in range(32):
        k1, r = lane % M, lane // M
        partner = ((32 - lane) & 31) if N == 512 else ((lane & ~(M - 1)) + ((M - k1) & (M - 1)))
        assert partner // M == r
        pk1 = partner % M
        for ab in range(6):
            v, pvv = X[(lane, ab)], X[(partner, ab)]
            for i in range(NH // M + 1):
                zm = pvv[(16 - i) & 15] if pk1 == 0 else pvv[15 - i]
                kk = k1 + M * i
                if kk <= NH:
                    sm, df = v[i] + zm, v[i] - zm
                    out[r, 2 * ab, kk] = sm.real + 1j * df.imag
                    out[r, 2 * ab + 1, kk] = sm.imag - 1j * df.real
    return out


def direct_products(N, U, V):
    R, NH = 512 // N, N // 2
    out = np.zeros((R, 12, NH + 1), complex)
    for r in range(R):
        zs = [np.fft.ifft(np.array([pack(U[r, c], V[r, c], x, N) for x in range(N)])) * N for c in range(3)]
        for ab, (ca, cb) in enumerate([(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]):
            Xf = np.fft.fft(zs[ca].real * zs[cb].real + 1j * zs[ca].imag * zs[cb].imag)
            for k in range(NH + 1):
                Zk, Zm = Xf[k], Xf[(N - k) % N]
                out[r, 2 * ab, k] = (Zk + np.conj(Zm)) / 2
                out[r, 2 * ab + 1, k] = (Zk - np.conj(Zm)) / 2j
    return out


def half_rows(N, seed):
    R, NH = 512 // N, N // 2
    rng = np.random.default_rng(seed)
    U = rng.standard_normal((R, 3, NH + 1)) + 1j * rng.standard_normal((R, 3, NH + 1))
    V = rng.standard_normal((R, 3, NH + 1)) + 1j * rng.standard_normal((R, 3, NH + 1))
    return U, V


@pytest.mark.parametrize("N", [128, 256, 512])
def test_product_pass_layout(N):
    U, V = half_rows(N, N)
    got, ref = products_stage(Layout(N), U, V), direct_products(N, U, V)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("N", [128, 256, 512])
def test_diagnostic_mode_layout(N):
    """Fields 0..2 are u_0..u_2 on one grid; the two sequences u_0 + i u_1 and u_2 (+ i 0)."""
    lay = Layout(N)
    R = lay.R
    F, _ = half_rows(N, N + 1)
    U = np.zeros_like(F)
    V = np.zeros_like(F)
    U[:, 0], V[:, 0], U[:, 1] = F[:, 0], F[:, 1], F[:, 2]  # V[:, 1] = 0: u_2 alone
    z = inverse_stages(lay, U, V, 2)
    for r in range(R):
        es, vm = 0.0, 0.0
        for lane in range(32):
            for p in range(lay.MP):
                if lay.row_b(lane, p) != r:
                    continue
                a, b = z[(lane, p, 0)], z[(lane, p, 1)]
                s2 = a.real ** 2 + a.imag ** 2 + b.real ** 2
                es, vm = es + 0.5 * s2.sum(), max(vm, s2.max())
        u = [np.fft.irfft(np.where(np.arange(N // 2 + 1) == 0, F[r, c].real, F[r, c]), n=N) * N for c in range(3)]
        # irfft takes only the real part at 0 and N/2, as the packing does
        s2 = u[0] ** 2 + u[1] ** 2 + u[2] ** 2
        assert abs(es - 0.5 * s2.sum()) <= 1e-12 * 0.5 * s2.sum()
        assert abs(vm - s2.max()) <= 1e-12 * s2.max()
