"""Encrypted 2-D FFT of an S x S image (S = 4^k) packed into two ciphertexts,
built from radix-4 diagonal-rotation stages (eblas/prepared_radix4_fft256.rs,
the R16.6b.3 decimation-in-time schedule of tests/r16_6b3_fft256_four_stage.rs:38-64).

Packing: ring degree N = S^2, N/2 = S^2/2 slots per ciphertext; image row R
(in base-4 digit-reversed order) lives in ciphertext R // (S/2) at slots
(R % (S/2)) * S .. + S - 1, columns also digit-reversed. The transform is
k row stages (spans 4 .. S slots inside every row), k - 1 column stages inside
each ciphertext (spans 4 .. S/4 rows, offsets in multiples of S slots) and one
column stage of span S rows across the two ciphertexts (offsets 0 and
+-N/4 slots, which are one Galois element). Every stage multiplies by its
diagonals encoded at the scale of the modulus it then rescales away, so the
ciphertext scale is unchanged; the output holds the 2-D DFT (sign -1) in
natural order.

The diagonals are public: they are built in FP64 on the host, encoded on the
GPU (ckks_encode) and transformed (ckks_ntt_forward) once per level.
"""
import numpy as np

from . import KeySwitchKey, encode, fft_stage, fft_stage_multi


def _root(n, e):
    return np.exp(-2j * np.pi * np.asarray(e, dtype=np.float64) / n)


def reverse_base4(i, digits):
    r = 0
    for _ in range(digits):
        r = r * 4 + i % 4
        i //= 4
    return r


def pack_image(img):
    """S x S real image -> two slot vectors (base-4 digit-reversed rows and columns)."""
    S = img.shape[0]
    k = int(round(np.log(S) / np.log(4)))
    assert 4 ** k == S and img.shape == (S, S)
    rev = np.array([reverse_base4(i, k) for i in range(S)])
    x = img[np.ix_(rev, rev)].astype(np.complex128)
    half = S // 2
    return np.stack([x[:half].reshape(-1), x[half:].reshape(-1)])


def unpack_spectrum(slots):
    """two slot vectors -> S x S spectrum in natural order."""
    S = int(round(np.sqrt(2 * slots.shape[-1])))
    return np.concatenate([slots[0].reshape(S // 2, S), slots[1].reshape(S // 2, S)])


def stage_diagonals(slots, span, unit):
    """Radix-4 DIT stage of span `span` elements, an element being `unit`
    consecutive slots: {offset: diagonal}, out[i] = sum diag[i] * in[i + offset]."""
    quarter = span // 4
    i = np.arange(slots)
    e = i // unit
    within = e % span
    p, j = within // quarter, within % quarter
    diags = {}
    for qd in range(4):
        off = (j + qd * quarter - within) * unit
        coef = _root(span, qd * j) * _root(4, p * qd)
        for o in np.unique(off):
            d = diags.setdefault(int(o), np.zeros(slots, np.complex128))
            m = off == o
            d[m] = coef[m]
    return dict(sorted(diags.items()))


def cross_stage_terms(S):
    """Last column stage (span S rows) across the two ciphertexts: a list of
    (output ct, input ct, rotated?, diagonal)."""
    half = S // 2
    slots = S * half
    i = np.arange(slots)
    lr = i // S  # local row
    jj = lr % (S // 4)
    terms = []
    for a in range(2):
        p = 2 * a + lr // (S // 4)
        for b in range(2):
            for rotated in (0, 1):
                d = np.zeros(slots, np.complex128)
                for qd in (2 * b, 2 * b + 1):
                    sel = (qd % 2 != p % 2) if rotated else (qd % 2 == p % 2)
                    coef = _root(S, qd * jj) * _root(4, p * qd)
                    d[sel] = coef[sel]
                terms.append((a, b, rotated, d))
    return terms


class Fft2Plan:
    """Keys and NTT-prepared diagonals of every stage, starting at Q-prefix
    level `level` (needs level >= 2 k + 1)."""

    def __init__(self, ctx, S, level, secret, base_log=32, seed=7000, keygen=None):
        import torch
        self.ctx, self.S = ctx, S
        k = int(round(np.log(S) / np.log(4)))
        assert 4 ** k == S and ctx.n == S * S and level >= 2 * k + 1
        self.k = k
        slots = ctx.n // 2
        keygen = keygen or (lambda lvl, e, sd: KeySwitchKey.hybrid_generate(ctx, lvl, base_log, e, secret, sd))
        self.stages = []
        lvl, sd = level, seed
        plan = [(4 ** (t + 1), 1) for t in range(k)] + [(4 ** (t + 1), S) for t in range(k - 1)]
        for span, unit in plan:
            diags = stage_diagonals(slots, span, unit)
            offs = [o for o in diags if o != 0]
            exps = [ctx.rotation_exponent_left(o) if o > 0 else ctx.rotation_exponent_right(-o) for o in offs]
            keys = [keygen(lvl, e, sd + i) for i, e in enumerate(exps)]
            sd += len(keys)
            plain_scale = float(ctx.q[lvl - 1])
            vecs = np.stack([diags[o] for o in offs] + [diags[0]])
            pt = encode(ctx, vecs, lvl, plain_scale)
            ctx.ntt_forward(pt)
            self.stages.append(("single", lvl, keys, pt))
            lvl -= 1
        terms = cross_stage_terms(S)
        e = ctx.rotation_exponent_left(slots // 2)
        key = keygen(lvl, e, sd)
        plain_scale = float(ctx.q[lvl - 1])
        pt = encode(ctx, np.stack([t[3] for t in terms]), lvl, plain_scale)
        ctx.ntt_forward(pt)
        tl = [(a, b, 0 if rot else 1) for a, b, rot, _ in terms]
        self.stages.append(("cross", lvl, [key], pt, tl))
        self.out_level = lvl - 1
        self.keys_bytes = None
        self._cross = {}  # images -> (terms, diagonals) of the cross stage over every image at once

    def _cross_batch(self, n_img):
        """The cross stage's terms and diagonals for n_img images in one call:
        image i's terms act on ciphertexts 2 i, 2 i + 1 with the same diagonals,
        so one hoisted rotation group covers every image (one key-switch MAC
        instead of one per image; the same words)."""
        import torch
        if n_img not in self._cross:
            _, _, _, pt, tl = self.stages[-1]
            terms = [(a + 2 * i, b + 2 * i, key) for i in range(n_img) for (a, b, key) in tl]
            self._cross[n_img] = (terms, torch.cat([pt] * n_img) if n_img > 1 else pt)
        return self._cross[n_img]

    def apply(self, cts, stream=None):
        """cts [n_images][2][2][level][N] -> [n_images][2][2][out_level][N]."""
        import torch
        n_img = cts.shape[0]
        cur = cts.reshape((n_img * 2,) + tuple(cts.shape[2:]))
        for st in self.stages:
            if st[0] == "single":
                cur = fft_stage(self.ctx, st[2], st[3], cur, identity=True, stream=stream)
            else:
                terms, diags = self._cross_batch(n_img)
                cur = fft_stage_multi(self.ctx, st[2], terms, diags, cur, 2 * n_img, stream=stream)
        return cur.reshape((n_img, 2) + tuple(cur.shape[1:]))
