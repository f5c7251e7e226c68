// Body of the float3 toolkit, included three times by vecmath.h: with plain
// operators (namespace qm: the compiler may contract a*b+c into an FMA),
// with explicitly rounded operations (namespace qs: every multiply, add and
// divide rounds separately, as in the CPU oracle, whatever the compilation
// flags), and with plain operators plus the approximate reciprocal square
// root and division (namespace qf, the approximate-math tracer build).  QR
// is the reciprocal square root, QRU the same for arguments of unit scale.  No include guard on purpose.



QM_HD float3 v3(float x, float y, float z) { return make_float3(x, y, z); }
QM_HD float3 add(float3 a, float3 b) { return make_float3(QA(a.x, b.x), QA(a.y, b.y), QA(a.z, b.z)); }
QM_HD float3 sub(float3 a, float3 b) { return make_float3(QS(a.x, b.x), QS(a.y, b.y), QS(a.z, b.z)); }
QM_HD float3 neg(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
QM_HD float3 mul(float3 a, float s) { return make_float3(QM(a.x, s), QM(a.y, s), QM(a.z, s)); }
QM_HD float3 adds(float3 a, float s) { return make_float3(QA(a.x, s), QA(a.y, s), QA(a.z, s)); }
QM_HD float3 subs(float3 a, float s) { return make_float3(QS(a.x, s), QS(a.y, s), QS(a.z, s)); }
QM_HD float3 cdiv(float3 a, float3 b) { return make_float3(QD(a.x, b.x), QD(a.y, b.y), QD(a.z, b.z)); }
// float3 / scalar goes through one reciprocal, as in the reference operator/.
QM_HD float3 divs(float3 a, float s) { float inv = QD(1.0f, s); return mul(a, inv); }
QM_HD float dot(float3 a, float3 b) { return QA(QA(QM(a.x, b.x), QM(a.y, b.y)), QM(a.z, b.z)); }
QM_HD float3 cross(float3 a, float3 b) {
  return make_float3(QS(QM(a.y, b.z), QM(a.z, b.y)), QS(QM(a.z, b.x), QM(a.x, b.z)), QS(QM(a.x, b.y), QM(a.y, b.x)));
}
QM_HD float rlen(float d) { return QR(d); }
QM_HD float length(float3 v) { return sqrtf(dot(v, v)); }
QM_HD float3 normalize(float3 v) { float inv = rlen(dot(v, v)); return mul(v, inv); }
// normalize for vectors of unit scale (squared length in [2^-125, 2^125) or
// NaN): the same value without the reciprocal square root's range test (QRU).
QM_HD float3 normalize_unit(float3 v) { float inv = QRU(dot(v, v)); return mul(v, inv); }
QM_HD float3 reflect(float3 i, float3 n) { return sub(i, mul(mul(n, 2.0f), dot(n, i))); }

QM_HD float dot2(float2 a, float2 b) { return QA(QM(a.x, b.x), QM(a.y, b.y)); }
QM_HD float length2(float2 v) { return sqrtf(dot2(v, v)); }
QM_HD float2 normalize2(float2 v) {
  float inv = rlen(dot2(v, v));
  return make_float2(QM(v.x, inv), QM(v.y, inv));
}

// Truncating float3 -> int3 (the reference's make_int3(float3) truncates
// toward zero, Util/vector_arithmetic.cuh:571-574).
QM_HD int3 trunc3(float3 a) { return make_int3(int(a.x), int(a.y), int(a.z)); }

// Orthonormal frame aligned with a normal: the columns (u, n, v) map local
// (x, y, z) to world.  `flip` selects the focus-flat variant that negates u
// and v when n.z < 0 (Scene/DataStructure/Heliostat/FocusFlatRectangleHelio.cuh:16-46);
// the plain variant is Util/global_function.cuh:19-36.
using Frame = ::qm_frame::Frame;

QM_HD Frame make_frame(float3 n, bool flip) {
  Frame f;
  f.n = n;
  f.identity = qm_below_eps(fabsf(n.x)) && qm_below_eps(fabsf(n.z));
  if (f.identity) {
    f.u = make_float3(1.f, 0.f, 0.f);
    f.v = make_float3(0.f, 0.f, 1.f);
    return f;
  }
  float3 u = normalize(cross(make_float3(0.0f, 1.0f, 0.0f), n));
  float3 v = normalize(cross(u, n));
  if (flip && n.z < 0) {
    u = neg(u);
    v = neg(v);
  }
  f.u = u;
  f.v = v;
  return f;
}

QM_HD float3 to_world(const Frame& f, float3 d) {
  if (f.identity) return d;
  return make_float3(QA(QA(QM(d.x, f.u.x), QM(d.y, f.n.x)), QM(d.z, f.v.x)),
                     QA(QA(QM(d.x, f.u.y), QM(d.y, f.n.y)), QM(d.z, f.v.y)),
                     QA(QA(QM(d.x, f.u.z), QM(d.y, f.n.z)), QM(d.z, f.v.z)));
}

QM_HD float3 rotate_to(float3 d, float3 n, bool flip) { return to_world(make_frame(n, flip), d); }

// Yaw-only rotation of a rectangle receiver vertex (Util/global_function.cuh:51-59).
QM_HD float3 rotate_y(float3 p, float3 old_dir, float3 new_dir) {
  int s = (cross(old_dir, new_dir).y > 0) ? 1 : -1;
  float c = dot(old_dir, new_dir);
  float sn = QM((float)s, sqrtf(QS(1.0f, QM(c, c))));
  return make_float3(QA(QM(c, p.x), QM(sn, p.z)), p.y, QA(QM(-sn, p.x), QM(c, p.z)));
}

// Ray / parallelogram test (Util/global_function.cuh:101-136) with the two
// edges supplied precomputed: ab = B - A and ac = C - A are formed exactly as
// the reference forms them inside the test, so results are unchanged.
QM_HD bool ray_parallelogram(float3 orig, float3 dir, float3 a, float3 ab, float3 ac,
                             float& t, float& u, float& v) {
  float3 p = cross(dir, ac);
  float det = dot(ab, p);
  if (qm_below_eps(fabsf(det))) return false;
  float3 tv = sub(orig, a);
  u = QD(dot(tv, p), det);
  if (u < 0 || u > 1) return false;
  float3 q = cross(tv, ab);
  v = QD(dot(dir, q), det);
  if (v < 0 || v > 1) return false;
  t = QD(dot(ac, q), det);
  if (qm_below_eps(t)) return false;
  return true;
}

// Atmospheric attenuation and per-ray energy
// (QuasiMonteCarloRayTracing/Receiver/receiverIntersectionUtil.cuh:17-34).
QM_HD float eta_atmosphere(float d) {
  if (d <= 1000.0f) return QA(QS(0.99331f, QM(0.0001176f, d)), QM(QM(QM(1.97f, 1e-8f), d), d));
  return expf(QM(-0.0001106f, d));
}

QM_HD float ray_energy(float distance, float3 dir, float3 normal, float factor) {
  return QM(QM(fabsf(dot(dir, normal)), eta_atmosphere(distance)), factor);
}

