"""threefry2x32 and the jax.random key/normal construction, in NumPy uint32.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Third-party algorithm on the path: JAX 0.10.2 (prolix uv.lock:915-1006) draws
the Langevin noise with ``jax.random.split`` and ``jax.random.normal``
(prolix physics/settle.py:2077-2087, batched_simulate.py:281-282).  JAX is
not installed here, so its published algorithm is restated:

* threefry2x32 with 20 rounds (Salmon, Moraes, Dror, Shaw, "Parallel random
  numbers: as easy as 1, 2, 3", SC'11): rotations (13,15,26,6),(17,29,16,24),
  key-schedule parity 0x1BD11BDA, a key injection after every four rounds.
  Pinned by the Random123 known-answer vectors in the tests.
* ``split`` and ``random_bits`` in the partitionable layout (JAX's default
  since 0.5): output element i of a shape is threefry(key, (hi32(i),
  lo32(i))); a 32-bit draw is the XOR of the two output words; ``split(key,
  n)`` returns the word pairs themselves.  The older layout (a single iota
  counter split in halves) is kept as ``partitionable=False``.
* ``uniform`` in float32: (bits >> 9) | 0x3F800000 reinterpreted, minus 1,
  scaled to [nextafter(-1, 0), 1) and clamped below; ``normal`` =
  sqrt(2) * erfinv(u).
* erfinv in float32 follows Giles, "Approximating the erfinv function"
  (GPU Computing Gems Jade, 2011), single-precision branch: w = -log(1-x^2),
  w < 5: polynomial in (w - 2.5); else polynomial in (sqrt(w) - 3); the
  coefficients are the ones published in that paper.  log(1-x^2) is taken
  as log1p(-x^2) with this project's own float32 log1p (below), computed
  with the same operation order as the CUDA kernel so the two agree
  bit-for-bit.  Whether XLA's erf_inv rounds identically is not pinned
  ("parity unpinned"): no JAX output is available here.
"""

from __future__ import annotations

import numpy as np

U32 = np.uint32
F32 = np.float32
ROT = (13, 15, 26, 6, 17, 29, 16, 24)
KS_PARITY = 0x1BD11BDA


def _rotl(x, r):
  r = U32(r)
  return (x << r) | (x >> U32(32 - int(r)))


def threefry2x32(k0, k1, x0, x1):
  """Vectorised Threefry-2x32-20 on uint32 arrays."""
  with np.errstate(over="ignore"):
    k0 = np.asarray(k0, U32)
    k1 = np.asarray(k1, U32)
    ks = (k0, k1, k0 ^ k1 ^ U32(KS_PARITY))
    x0 = np.asarray(x0, U32) + ks[0]
    x1 = np.asarray(x1, U32) + ks[1]
    for r in range(20):
      x0 = x0 + x1
      x1 = _rotl(x1, ROT[r % 8])
      x1 = x1 ^ x0
      if r % 4 == 3:
        s = (r + 1) // 4
        x0 = x0 + ks[s % 3]
        x1 = x1 + ks[(s + 1) % 3] + U32(s)
  return x0, x1


def prng_key(seed: int):
  """jax.random.PRNGKey(seed) for the threefry implementation: (hi32, lo32)."""
  seed = int(seed) & 0xFFFFFFFFFFFFFFFF
  return np.array([(seed >> 32) & 0xFFFFFFFF, seed & 0xFFFFFFFF], dtype=U32)


def split(key, num=2, partitionable=True):
  """jax.random.split(key, num) -> (num, 2) uint32."""
  key = np.asarray(key, U32)
  if partitionable:
    i = np.arange(num, dtype=np.uint64)
    a, b = threefry2x32(key[0], key[1], (i >> np.uint64(32)).astype(U32),
                        (i & np.uint64(0xFFFFFFFF)).astype(U32))
    return np.stack([a, b], axis=1)
  cnt = np.arange(2 * num, dtype=U32)
  a, b = threefry2x32(key[0], key[1], cnt[:num], cnt[num:])
  return np.concatenate([a, b]).reshape(num, 2)


def random_bits32(key, count, partitionable=True):
  """32-bit random words for a flat array of ``count`` elements."""
  key = np.asarray(key, U32)
  if partitionable:
    i = np.arange(count, dtype=np.uint64)
    a, b = threefry2x32(key[0], key[1], (i >> np.uint64(32)).astype(U32),
                        (i & np.uint64(0xFFFFFFFF)).astype(U32))
    return a ^ b
  half = (count + 1) // 2
  cnt = np.arange(2 * half, dtype=U32)
  a, b = threefry2x32(key[0], key[1], cnt[:half], cnt[half:])
  return np.concatenate([a, b])[:count]


LO = np.nextafter(F32(-1.0), F32(0.0))


def uniform_pm1(bits):
  """float32 uniform on [nextafter(-1, 0), 1) from 32-bit words."""
  fb = (np.asarray(bits, U32) >> U32(9)) | U32(0x3F800000)
  f = fb.view(F32) - F32(1.0)
  span = F32(1.0) - LO  # rounds to 2.0f
  return np.maximum(LO, f * span + LO)


def log1p_f32(x):
  """float32 log(1 + x) for x in (-1, 0], own construction.

  1 + x = m * 2^e with m in [sqrt(1/2), sqrt(2)); log(m) = 2 atanh(s) with
  s = (m - 1) / (m + 1), |s| <= 0.1716, summed as the odd Taylor series of
  atanh to s^15 (|remainder| < 2e-13); e * ln 2 split in a hi/lo pair.  For
  |x| < 2^-12 the series log1p(x) = x - x^2/2 + x^3/3 is used directly.
  Every step is a single float32 operation, so the result is reproducible.
  """
  x = np.asarray(x, F32)
  one = F32(1.0)
  u = one + x
  # exact correction of the rounding in 1 + x
  c = (x - (u - one)) / u
  bits = u.view(U32).astype(np.int64)
  e = ((bits >> 23) & 0xFF) - 127
  mbits = (bits & 0x7FFFFF) | 0x3F800000
  m = mbits.astype(U32).view(F32)
  big = m > F32(1.4142135)
  m = np.where(big, m * F32(0.5), m).astype(F32)
  e = np.where(big, e + 1, e)
  s = (m - one) / (m + one)
  s2 = s * s
  p = F32(1.0 / 15.0)
  for k in (13, 11, 9, 7, 5, 3):
    p = p * s2 + F32(1.0 / k)
  p = p * s2
  lm = F32(2.0) * s + F32(2.0) * s * p
  ef = e.astype(F32)
  ln2_hi = F32(0.693145751953125)
  ln2_lo = F32(1.428606765330187e-06)
  r = ef * ln2_hi + (lm + (ef * ln2_lo + c))
  small = np.abs(x) < F32(2.0 ** -12)
  rs = x * (one - x * (F32(0.5) - x * F32(1.0 / 3.0)))
  return np.where(small, rs, r).astype(F32)


# Giles (2011), single-precision erfinv coefficients, highest order first
_W_LT5 = (2.81022636e-08, 3.43273939e-07, -3.5233877e-06, -4.39150654e-06,
          0.00021858087, -0.00125372503, -0.00417768164, 0.246640727, 1.50140941)
_W_GE5 = (-0.000200214257, 0.000100950558, 0.00134934322, -0.00367342844,
          0.00573950773, -0.0076224613, 0.00943887047, 1.00167406, 2.83297682)


def erfinv_f32(x):
  x = np.asarray(x, F32)
  w = -log1p_f32(-(x * x))
  lt = w < F32(5.0)
  wa = (w - F32(2.5)).astype(F32)
  wb = (np.sqrt(np.maximum(w, F32(0.0))).astype(F32) - F32(3.0)).astype(F32)
  pa = np.full_like(x, F32(_W_LT5[0]))
  pb = np.full_like(x, F32(_W_GE5[0]))
  for ca, cb in zip(_W_LT5[1:], _W_GE5[1:]):
    pa = (F32(ca) + pa * wa).astype(F32)
    pb = (F32(cb) + pb * wb).astype(F32)
  p = np.where(lt, pa, pb)
  res = (p * x).astype(F32)
  return np.where(np.abs(x) == F32(1.0), x * np.finfo(F32).max, res).astype(F32)


def normal_f32(key, count, partitionable=True):
  """jax.random.normal(key, (count,), float32) restated."""
  u = uniform_pm1(random_bits32(key, count, partitionable))
  return (F32(np.sqrt(2.0)) * erfinv_f32(u)).astype(F32)
