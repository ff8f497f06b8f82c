"""The few glm 0.9.6 float operations the reference's glTF loader uses, restated in numpy float32
with glm's evaluation order, so that a scene loaded here carries the reference's matrices and
camera bit for bit (src/scene/scene_load_gltf.cpp:243-300, 465-500).

Matrices are 4x4 float32 arrays indexed m[column][row], glm's layout. glm is the header-only
math library the reference vendors (external/include/glm); its formulas are restated here:
  * mat4 * mat4: column i = ((A0 b0 + A1 b1) + A2 b2) + A3 b3 with b = column i of the right;
  * translate(m, v): column 3 = ((m0 v0 + m1 v1) + m2 v2) + m3;
  * scale(m, v): columns 0..2 scaled by v;
  * mat4_cast(quat): the products qxx .. qwz, then 1 - 2 (qyy + qzz) etc.;
  * inverse: the cofactor form with factors Coef00..Coef23, determinant (x + y) + (z + w) of
    column 0 times the first row of the adjugate, and the adjugate multiplied by 1 / det;
  * inverseTranspose: the cofactor form with SubFactor00..18, divided by its determinant;
  * normalize: v * (1 / sqrt(dot(v, v))), dot = (x x + y y) + z z.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def identity() -> np.ndarray:
    return np.eye(4, dtype=f32)


def mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    out = np.empty((4, 4), f32)
    for i in range(4):
        out[i] = ((a[0] * b[i][0] + a[1] * b[i][1]) + a[2] * b[i][2]) + a[3] * b[i][3]
    return out


def translate(m: np.ndarray, v) -> np.ndarray:
    v = np.asarray(v, dtype=np.float64).astype(f32)
    out = m.copy()
    out[3] = ((m[0] * v[0] + m[1] * v[1]) + m[2] * v[2]) + m[3]
    return out


def scale(m: np.ndarray, v) -> np.ndarray:
    v = np.asarray(v, dtype=np.float64).astype(f32)
    out = m.copy()
    for c in range(3):
        out[c] = m[c] * v[c]
    return out


def mat4_cast(w, x, y, z) -> np.ndarray:
    w, x, y, z = f32(w), f32(x), f32(y), f32(z)
    qxx, qyy, qzz = x * x, y * y, z * z
    qxz, qxy, qyz = x * z, x * y, y * z
    qwx, qwy, qwz = w * x, w * y, w * z
    one, two = f32(1), f32(2)
    r = identity()
    r[0][0] = one - two * (qyy + qzz)
    r[0][1] = two * (qxy + qwz)
    r[0][2] = two * (qxz - qwy)
    r[1][0] = two * (qxy - qwz)
    r[1][1] = one - two * (qxx + qzz)
    r[1][2] = two * (qyz + qwx)
    r[2][0] = two * (qxz + qwy)
    r[2][1] = two * (qyz - qwx)
    r[2][2] = one - two * (qxx + qyy)
    return r


def inverse(m: np.ndarray) -> np.ndarray:
    m = np.asarray(m, f32)

    def c(a, b, cc, d, e, f, g, h):  # m[a][b] * m[cc][d] - m[e][f] * m[g][h]
        return m[a][b] * m[cc][d] - m[e][f] * m[g][h]

    coef00, coef02, coef03 = c(2, 2, 3, 3, 3, 2, 2, 3), c(1, 2, 3, 3, 3, 2, 1, 3), c(1, 2, 2, 3, 2, 2, 1, 3)
    coef04, coef06, coef07 = c(2, 1, 3, 3, 3, 1, 2, 3), c(1, 1, 3, 3, 3, 1, 1, 3), c(1, 1, 2, 3, 2, 1, 1, 3)
    coef08, coef10, coef11 = c(2, 1, 3, 2, 3, 1, 2, 2), c(1, 1, 3, 2, 3, 1, 1, 2), c(1, 1, 2, 2, 2, 1, 1, 2)
    coef12, coef14, coef15 = c(2, 0, 3, 3, 3, 0, 2, 3), c(1, 0, 3, 3, 3, 0, 1, 3), c(1, 0, 2, 3, 2, 0, 1, 3)
    coef16, coef18, coef19 = c(2, 0, 3, 2, 3, 0, 2, 2), c(1, 0, 3, 2, 3, 0, 1, 2), c(1, 0, 2, 2, 2, 0, 1, 2)
    coef20, coef22, coef23 = c(2, 0, 3, 1, 3, 0, 2, 1), c(1, 0, 3, 1, 3, 0, 1, 1), c(1, 0, 2, 1, 2, 0, 1, 1)
    fac0 = np.array([coef00, coef00, coef02, coef03], f32)
    fac1 = np.array([coef04, coef04, coef06, coef07], f32)
    fac2 = np.array([coef08, coef08, coef10, coef11], f32)
    fac3 = np.array([coef12, coef12, coef14, coef15], f32)
    fac4 = np.array([coef16, coef16, coef18, coef19], f32)
    fac5 = np.array([coef20, coef20, coef22, coef23], f32)
    vec0 = np.array([m[1][0], m[0][0], m[0][0], m[0][0]], f32)
    vec1 = np.array([m[1][1], m[0][1], m[0][1], m[0][1]], f32)
    vec2 = np.array([m[1][2], m[0][2], m[0][2], m[0][2]], f32)
    vec3 = np.array([m[1][3], m[0][3], m[0][3], m[0][3]], f32)
    inv0 = (vec1 * fac0 - vec2 * fac1) + vec3 * fac2
    inv1 = (vec0 * fac0 - vec2 * fac3) + vec3 * fac4
    inv2 = (vec0 * fac1 - vec1 * fac3) + vec3 * fac5
    inv3 = (vec0 * fac2 - vec1 * fac4) + vec2 * fac5
    sa = np.array([1, -1, 1, -1], f32)
    sb = np.array([-1, 1, -1, 1], f32)
    inv = np.stack([inv0 * sa, inv1 * sb, inv2 * sa, inv3 * sb]).astype(f32)
    row0 = np.array([inv[0][0], inv[1][0], inv[2][0], inv[3][0]], f32)
    dot0 = m[0] * row0
    dot1 = (dot0[0] + dot0[1]) + (dot0[2] + dot0[3])
    return (inv * (f32(1) / dot1)).astype(f32)


def inverse_transpose(m: np.ndarray) -> np.ndarray:
    m = np.asarray(m, f32)

    def s(a, b, cc, d, e, f, g, h):
        return m[a][b] * m[cc][d] - m[e][f] * m[g][h]

    sf = [s(2, 2, 3, 3, 3, 2, 2, 3), s(2, 1, 3, 3, 3, 1, 2, 3), s(2, 1, 3, 2, 3, 1, 2, 2), s(2, 0, 3, 3, 3, 0, 2, 3),
          s(2, 0, 3, 2, 3, 0, 2, 2), s(2, 0, 3, 1, 3, 0, 2, 1), s(1, 2, 3, 3, 3, 2, 1, 3), s(1, 1, 3, 3, 3, 1, 1, 3),
          s(1, 1, 3, 2, 3, 1, 1, 2), s(1, 0, 3, 3, 3, 0, 1, 3), s(1, 0, 3, 2, 3, 0, 1, 2), s(1, 1, 3, 3, 3, 1, 1, 3),
          s(1, 0, 3, 1, 3, 0, 1, 1), s(1, 2, 2, 3, 2, 2, 1, 3), s(1, 1, 2, 3, 2, 1, 1, 3), s(1, 1, 2, 2, 2, 1, 1, 2),
          s(1, 0, 2, 3, 2, 0, 1, 3), s(1, 0, 2, 2, 2, 0, 1, 2), s(1, 0, 2, 1, 2, 0, 1, 1)]

    def t(sign, a, i, b, j, cc, k):  # sign * ((a*sf[i] - b*sf[j]) + cc*sf[k])
        v = (a * sf[i] - b * sf[j]) + cc * sf[k]
        return v if sign > 0 else -v

    r = np.empty((4, 4), f32)
    r[0][0] = t(1, m[1][1], 0, m[1][2], 1, m[1][3], 2)
    r[0][1] = t(-1, m[1][0], 0, m[1][2], 3, m[1][3], 4)
    r[0][2] = t(1, m[1][0], 1, m[1][1], 3, m[1][3], 5)
    r[0][3] = t(-1, m[1][0], 2, m[1][1], 4, m[1][2], 5)
    r[1][0] = t(-1, m[0][1], 0, m[0][2], 1, m[0][3], 2)
    r[1][1] = t(1, m[0][0], 0, m[0][2], 3, m[0][3], 4)
    r[1][2] = t(-1, m[0][0], 1, m[0][1], 3, m[0][3], 5)
    r[1][3] = t(1, m[0][0], 2, m[0][1], 4, m[0][2], 5)
    r[2][0] = t(1, m[0][1], 6, m[0][2], 7, m[0][3], 8)
    r[2][1] = t(-1, m[0][0], 6, m[0][2], 9, m[0][3], 10)
    r[2][2] = t(1, m[0][0], 11, m[0][1], 9, m[0][3], 12)
    r[2][3] = t(-1, m[0][0], 8, m[0][1], 10, m[0][2], 12)
    r[3][0] = t(-1, m[0][1], 13, m[0][2], 14, m[0][3], 15)
    r[3][1] = t(1, m[0][0], 13, m[0][2], 16, m[0][3], 17)
    r[3][2] = t(-1, m[0][0], 14, m[0][1], 16, m[0][3], 18)
    r[3][3] = t(1, m[0][0], 15, m[0][1], 17, m[0][2], 18)
    det = ((m[0][0] * r[0][0] + m[0][1] * r[0][1]) + m[0][2] * r[0][2]) + m[0][3] * r[0][3]
    return (r / det).astype(f32)


def normalize(v) -> np.ndarray:
    v = np.asarray(v, f32)
    d = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]
    return v * (f32(1) / np.sqrt(d))
