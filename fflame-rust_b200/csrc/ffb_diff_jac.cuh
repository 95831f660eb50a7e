// ffb_diff_jac.cuh -- analytic Jacobians of the variation bodies for the
// differentiable render, compiled by NVRTC after ffb_device.cuh (whose
// bodies give the values) and before the generated ffb_dnormal.

// Variation Jacobians: J = (dVx/dx, dVx/dy, dVy/dx, dVy/dy) at (x, y).
// Derived from the bodies above; the value comes from the body itself.
__device__ __forceinline__ float4 dj_linear(float, float) { return make_float4(1.f, 0.f, 0.f, 1.f); }
__device__ __forceinline__ float4 dj_sinusoidal(float x, float y) { return make_float4(cosf(x), 0.f, 0.f, cosf(y)); }
__device__ __forceinline__ float4 dj_cylinder(float x, float) { return make_float4(cosf(x), 0.f, 0.f, 1.f); }
__device__ __forceinline__ float4 dj_spherical(float x, float y) {
    const float r2 = x * x + y * y + 1e-6f, i = 1.0f / r2, i2 = i * i;
    return make_float4(i - 2.f * x * x * i2, -2.f * x * y * i2, -2.f * x * y * i2, i - 2.f * y * y * i2);
}
__device__ __forceinline__ float4 dj_swirl(float x, float y) {
    const float r2 = x * x + y * y;
    float s, c;
    sincosf(r2, &s, &c);
    const float vx = x * s - y * c, vy = x * c + y * s;
    return make_float4(s + 2.f * x * vy, -c + 2.f * y * vy, c - 2.f * x * vx, s - 2.f * y * vx);
}
__device__ __forceinline__ float4 dj_horseshoe(float x, float y) {
    const float rho = sqrtf(x * x + y * y);
    if (!(rho > 0.f)) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float r = rho + 1e-6f, ir = 1.0f / r, ir2 = ir * ir;
    const float a = x * x - y * y, b = 2.f * x * y, ux = x / rho, uy = y / rho;
    return make_float4(2.f * x * ir - a * ir2 * ux, -2.f * y * ir - a * ir2 * uy, 2.f * y * ir - b * ir2 * ux, 2.f * x * ir - b * ir2 * uy);
}
__device__ __forceinline__ float4 dj_polar(float x, float y) {
    const float r2 = x * x + y * y, rho = sqrtf(r2);
    if (!(rho > 0.f)) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float k = 1.0f / (FFB_PI * r2);                   // th = atan2(x, y): dth = (y, -x) / r2
    return make_float4(y * k, -x * k, x / rho, y / rho);
}
__device__ __forceinline__ float4 dj_disc(float x, float y) {
    const float r2 = x * x + y * y, rho = sqrtf(r2);
    if (!(rho > 0.f)) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float tp = atan2f(x, y) / FFB_PI;
    float s, c;
    sincosf(FFB_PI * rho, &s, &c);
    const float k = 1.0f / (FFB_PI * r2);
    const float tpx = y * k, tpy = -x * k;                  // d(tp)
    const float prx = FFB_PI * x / rho, pry = FFB_PI * y / rho;   // d(pi r)
    return make_float4(tpx * s + tp * c * prx, tpy * s + tp * c * pry, tpx * c - tp * s * prx, tpy * c - tp * s * pry);
}
__device__ __forceinline__ float4 dj_ex(float x, float y) {
    const float r2 = x * x + y * y, r = sqrtf(r2);
    if (!(r > 0.f)) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float th = atan2f(y, x);
    float s0, c0, s1, c1;
    sincosf(th + r, &s0, &c0);                              // n0 = sin(th + r)
    sincosf(th - r, &s1, &c1);                              // n1 = cos(th - r)
    const float m0 = s0 * s0 * s0, m1 = c1 * c1 * c1;
    const float thx = -y / r2, thy = x / r2, rx = x / r, ry = y / r;
    const float dm0x = 3.f * s0 * s0 * c0 * (thx + rx), dm0y = 3.f * s0 * s0 * c0 * (thy + ry);
    const float dm1x = -3.f * c1 * c1 * s1 * (thx - rx), dm1y = -3.f * c1 * c1 * s1 * (thy - ry);
    return make_float4(rx * (m0 + m1) + r * (dm0x + dm1x), ry * (m0 + m1) + r * (dm0y + dm1y),
                       rx * (m0 - m1) + r * (dm0x - dm1x), ry * (m0 - m1) + r * (dm0y - dm1y));
}
__device__ __forceinline__ float4 dj_julia(float x, float y, float d) {
    const float r2 = x * x + y * y, r = sqrtf(r2);
    if (!(r > 0.f)) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float sr = sqrtf(r);
    const float ht = atan2f(y, x) / 2.0f + ((d < 0.5f) ? FFB_PI : 0.0f);
    float s, c;
    sincosf(ht, &s, &c);
    const float srx = x / (2.f * r * sr), sry = y / (2.f * r * sr);   // d sqrt(r)
    const float htx = -y / (2.f * r2), hty = x / (2.f * r2);          // d(th / 2)
    return make_float4(srx * c - sr * s * htx, sry * c - sr * s * hty, srx * s + sr * c * htx, sry * s + sr * c * hty);
}
__device__ __forceinline__ float4 dj_bubble(float x, float y) {
    const float rr = (x * x + y * y) / 4.0f + 1.0f, s = 1.0f / rr;
    const float k = -0.5f * s * s;                          // ds = k (x, y)
    return make_float4(s + x * k * x, x * k * y, y * k * x, s + y * k * y);
}
__device__ __forceinline__ float4 dj_curl(float x, float y, float c1, float c2) {
    // V = z / w with w = 1 + c1 z + c2 z^2 (holomorphic): V' = (1 - c2 z^2) / w^2.
    const float re = 1.0f + c1 * x + c2 * (x * x - y * y), im = c1 * y + 2.0f * c2 * x * y;
    const float nr = 1.0f - c2 * (x * x - y * y), ni = -2.0f * c2 * x * y;
    const float wr = re * re - im * im, wi = 2.0f * re * im;
    const float den = 1.0f / (wr * wr + wi * wi);
    const float a = (nr * wr + ni * wi) * den, b = (ni * wr - nr * wi) * den;
    return make_float4(a, -b, b, a);
}
