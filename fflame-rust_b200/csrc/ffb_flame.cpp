// ffb_flame.cpp -- parsing the `.fae` flame description and deriving the
// tables the kernels read.  See ffb_flame.hpp for the reference files.

#include "ffb_flame.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <random>

namespace ffb {

// The host restatements of the variations' `wgsl_init` (f32, the same
// operations): user parameters -> derived values.
namespace {
void derive_julian(const float* u, float* o) {                 // advanced.rs:467-473
    o[0] = u[1] / std::max(std::fabs(u[0]), 1e-30f) / 2.0f;
}
void derive_wedge(const float* u, float* o) {                  // extended.rs:273-281
    const float angle_rad = u[0] * 3.14159265358979f / 180.0f;
    o[0] = angle_rad;
    o[1] = 1.0f - angle_rad * u[2] * 0.15915494309189534f;
}
void derive_radial_blur(const float* u, float* o) {            // extended.rs:867-874
    const float half = u[0] * 3.14159265358979f / 360.0f;
    o[0] = std::sin(half);
    o[1] = std::cos(half);
}
void derive_perspective(const float* u, float* o) {            // simple_classics.rs:315-322
    const float ang = u[0] * 1.5707963267948966f;
    o[0] = std::sin(ang);
    o[1] = u[1] * std::cos(ang);
}

void derive_log(const float* u, float* o) {                    // advanced.rs (init_log)
    o[0] = 0.5f / std::log(std::max(u[0], 1.000001f));
}
void derive_escher(const float* u, float* o) {                 // advanced.rs (init_escher)
    const float beta = u[0] * 3.14159265358979f / 180.0f;
    o[0] = 0.5f * (1.0f + std::cos(beta));
    o[1] = 0.5f * std::sin(beta);
}
void derive_modulus(const float* u, float* o) {                // singleton_misc.rs (init_modulus)
    o[0] = 2.0f * u[0];
    o[1] = 2.0f * u[1];
}
void derive_curve(const float* u, float* o) {                  // erf_misc.rs (init_curve)
    o[0] = std::max(u[2] * u[2], 1e-20f);
    o[1] = std::max(u[3] * u[3], 1e-20f);
}

void derive_disc2(const float* u, float* o) {                  // heavy_init.rs (init_disc2)
    const float two_pi = 6.28318530717959f;
    const float twist = u[1];
    float sinadd = std::sin(twist), cosadd = std::cos(twist) - 1.0f;
    if (twist > two_pi) { const float k = 1.0f + twist - two_pi; cosadd *= k; sinadd *= k; }
    if (twist < -two_pi) { const float k = 1.0f + twist + two_pi; cosadd *= k; sinadd *= k; }
    o[0] = u[0] * 3.14159265358979f;
    o[1] = cosadd;
    o[2] = sinadd;
}
void derive_cpow(const float* u, float* o) {                   // advanced.rs (init_cpow)
    const float sp = u[2] == 0.0f ? 1e-30f : u[2];
    o[0] = 6.28318530717959f / sp;
    o[1] = u[0] / sp;
    o[2] = u[1] / sp;
}
void derive_oscilloscope(const float* u, float* o) {           // misc_extras2.rs (init_oscilloscope)
    o[0] = 6.28318530717959f * u[1];
}
void derive_wedge_julia(const float* u, float* o) {            // wedge_extended.rs (init_wedge_julia)
    const float sp = u[0] == 0.0f ? 1e-30f : u[0];
    o[0] = 1.0f - u[3] * u[2] * 0.15915494309189535f;
    o[1] = std::fabs(u[0]);
    o[2] = u[1] / sp * 0.5f;
}
void derive_wedge_sph(const float* u, float* o) {              // wedge_extended.rs (init_wedge_sph)
    o[0] = 1.0f - u[0] * u[2] * 0.15915494309189535f;
}

// f32 complex arithmetic in the operation order of shaders/core/complex.wgsl:20-69.
struct Cx { float x, y; };
Cx cadd(Cx a, Cx b) { return {a.x + b.x, a.y + b.y}; }
Cx csub(Cx a, Cx b) { return {a.x - b.x, a.y - b.y}; }
Cx cmul(Cx a, Cx b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
Cx cmulr(Cx a, float s) { return {a.x * s, a.y * s}; }
Cx cdiv(Cx a, Cx b) {
    const float d = b.x * b.x + b.y * b.y;
    const float sd = d < 1e-30f ? 1e-30f : d;
    const Cx n = cmul(a, Cx{b.x, -b.y});
    return {n.x / sd, n.y / sd};
}
Cx csq(Cx a) { return {a.x * a.x - a.y * a.y, 2.0f * a.x * a.y}; }
Cx csqrt(Cx a) {
    const float mag = std::sqrt(a.x * a.x + a.y * a.y);
    const float re = std::sqrt(std::fmax(0.5f * (mag + a.x), 0.0f));
    const float im = std::sqrt(std::fmax(0.5f * (mag - a.x), 0.0f));
    return {re, a.y >= 0.0f ? im : -im};
}

// klein_group's generator pair from its recipe (klein_group_misc.rs:82-225):
// mat_a then mat_b, each four complex entries as (re, im).
void derive_klein_group(const float* u, float* o) {
    const Cx zero{0, 0}, re1{1, 0}, re2{2, 0}, re4{4, 0}, im1{0, 1}, im2{0, 2}, im4{0, 4};
    const int recipe = (int)u[4];
    Cx a[4] = {re1, zero, zero, re1}, b[4] = {re1, zero, zero, re1};
    auto maskit_a = [&](Cx mu) {
        a[0] = cmul(cmulr(mu, -1.0f), im1);
        a[1] = cmulr(im1, -1.0f);
        a[2] = cmulr(im1, -1.0f);
        a[3] = zero;
    };
    // The trace-AB root both trace recipes share: (-bb - sqrt(bb^2 - 4 cc)) / 2.
    auto tr_ab = [&](Cx trA, Cx trB, Cx& tab, Cx& safe) {
        const Cx bb = cmulr(cmul(trA, trB), -1.0f);
        const Cx cc = cadd(csq(trA), csq(trB));
        const Cx disc = csqrt(csub(csq(bb), cmulr(cc, 4.0f)));
        tab = cmulr(csub(cmulr(bb, -1.0f), disc), 0.5f);
        safe = {std::fabs(tab.x) + std::fabs(tab.y) < 1e-15f ? 1e-15f : tab.x, tab.y};
    };
    if (recipe == 3) {                                   // Riley
        a[2] = {u[0], u[1]};
        b[1] = re2;
    } else if (recipe == 4) {                            // Riley, b1 given
        a[2] = {u[0], u[1]};
        b[1] = {u[2], u[3]};
    } else if (recipe == 1) {                            // Maskit mu
        maskit_a({u[0], u[1]});
        b[1] = re2;
    } else if (recipe == 5) {                            // Maskit mu, b1 given
        maskit_a({u[0], u[1]});
        b[1] = {u[2], u[3]};
    } else if (recipe == 6) {                            // Maskit-Leys: b1 = 2 cos(pi / n) + i b_im
        maskit_a({u[0], u[1]});
        const float safe_br = std::fabs(u[2]) < 1e-30f ? 1e-30f : u[2];
        b[1] = {2.0f * std::cos(3.14159265358979f / safe_br), u[3]};
    } else if (recipe == 2) {                            // Jorgensen
        const Cx trA{u[0], u[1]}, trB{u[2], u[3]};
        Cx tab, s;
        tr_ab(trA, trB, tab, s);
        a[0] = csub(trA, cdiv(trB, s)); a[1] = cdiv(trA, csq(s)); a[2] = trA; a[3] = cdiv(trB, s);
        b[0] = csub(trB, cdiv(trA, s)); b[1] = cmulr(cdiv(trB, csq(s)), -1.0f); b[2] = cmulr(trB, -1.0f); b[3] = cdiv(trA, s);
    } else {                                             // Grandma's parabolic commutator (0 and any other)
        const Cx trA{u[0], u[1]}, trB{u[2], u[3]};
        Cx tab, s;
        tr_ab(trA, trB, tab, s);
        const Cx z0 = cdiv(cmul(csub(tab, re2), trB), cadd(csub(cmul(trB, s), cmulr(trA, 2.0f)), cmul(s, im2)));
        a[0] = cmulr(trA, 0.5f);
        a[1] = cdiv(cadd(csub(cmul(trA, s), cmulr(trB, 2.0f)), im4), cmul(cadd(cmulr(s, 2.0f), re4), z0));
        a[2] = cdiv(cmul(csub(csub(cmul(trA, s), cmulr(trB, 2.0f)), im4), z0), csub(cmulr(s, 2.0f), re4));
        a[3] = cmulr(trA, 0.5f);
        b[0] = cmulr(csub(trB, im2), 0.5f);
        b[1] = cmulr(trB, 0.5f);
        b[2] = cmulr(trB, 0.5f);
        b[3] = cmulr(cadd(trB, im2), 0.5f);
    }
    for (int i = 0; i < 4; ++i) {
        o[2 * i] = a[i].x; o[2 * i + 1] = a[i].y;
        o[8 + 2 * i] = b[i].x; o[8 + 2 * i + 1] = b[i].y;
    }
}

// subflame_wf's placement rotation (subflame.wgsl:399-408): cos and sin of
// angle x 0.017453292519943295 in f32, taken once here instead of per call.
void derive_subflame(const float* u, float* o) {
    const float ang = u[2] * 0.017453292519943295f;
    o[0] = std::cos(ang);
    o[1] = std::sin(ang);
}
void derive_shift(const float* u, float* o) {                   // misc_2d.rs (init_shift)
    const float a = u[2] * 3.14159265358979f / 180.0f;
    o[0] = std::cos(a); o[1] = std::sin(a);
}
void derive_pressure_wave(const float* u, float* o) {           // misc_2d.rs (init_pressure_wave)
    const float tp = 6.28318530717959f;
    const float px = u[0] != 0.0f ? u[0] * tp : 1.0f, py = u[1] != 0.0f ? u[1] * tp : 1.0f;
    o[0] = px; o[1] = py; o[2] = 1.0f / px; o[3] = 1.0f / py;
}
void derive_spligon(const float* u, float* o) {                 // misc_2d.rs (init_spligon)
    const float s = u[0] == 0.0f ? 1e-30f : u[0], th = s / 6.28318530717959f;
    o[0] = th; o[1] = 1.0f / th; o[2] = 3.14159265358979f * u[1] / (-2.0f * s);
}
void derive_circus(const float* u, float* o) { o[0] = 1.0f / std::max(u[0], 1e-6f); }   // singleton_misc.rs (init_circus)
void derive_murl(const float* u, float* o) {                    // singleton_misc.rs (init_murl)
    float c = u[0];
    if (u[1] != 1.0f) { const float m = u[1] - 1.0f; c = c / (std::fabs(m) < 1e-30f ? 1e-30f : m); }
    o[0] = c; o[1] = u[1] * 0.5f; o[2] = c + 1.0f;
}
void derive_target(const float* u, float* o) { o[0] = 0.5f * u[2]; }                    // init_ports.rs (init_target)
void derive_bwraps(const float* u, float* o) {                  // extended.rs (init_bwraps)
    if (u[0] == 0.0f) { o[0] = o[1] = o[2] = 0.0f; return; }
    const float rad = 0.5f * (u[0] / (1.0f + u[1] * u[1])), g2 = (u[2] * u[2]) / (rad + 1e-6f) + 1e-6f;
    float mb = g2 * rad;
    mb = mb > 2.0f ? 1.0f : mb * (1.0f / ((mb * mb) / 4.0f + 1.0f));
    o[0] = g2; o[1] = rad * rad; o[2] = rad / mb;
}
void derive_hypershift2(const float* u, float* o) {             // apo_misc16.rs (init_hypershift2)
    const float pi = 3.14159265358979f, pi_2 = 1.5707963267948966f;
    const float p = std::fmax(u[0], 2.0f), q = std::fmax(u[1], 2.0f), pq = pi / q, pp = pi / p;
    const float spq = std::sin(pq), spp = std::sin(pp);
    const float shift = std::sin(pi_2 - pq - pp) / std::sqrt(std::fmax(1.0f - spq * spq - spp * spp, 1e-30f));
    const float s_p2pp = std::sin(pi_2 + pp), r_inner = s_p2pp * s_p2pp / (spq * spq) - 1.0f;
    const float scale2 = 1.0f / std::sqrt(std::fmax(r_inner, 1e-30f)) * (s_p2pp / spq - 1.0f);
    o[0] = shift; o[1] = scale2; o[2] = 1.0f - shift * shift; o[3] = 1.0f / p;
}
void derive_hypertile(const float* u, float* o) {               // hypertile.rs (init_hypertile)
    const float pi = 3.14159265358979f, pa = 2.0f * pi / u[0], qa = 2.0f * pi / u[1];
    const float ri = (1.0f - std::cos(pa)) / (std::cos(pa) + std::cos(qa)) + 1.0f;
    const float r = ri > 0.0f ? 1.0f / std::sqrt(ri) : 1.0f, a = u[2] * pa;
    o[0] = r * std::cos(a); o[1] = r * std::sin(a);
}
void derive_hypertile1(const float* u, float* o) {              // hypertile.rs (init_hypertile1)
    const float pi = 3.14159265358979f, pa = 2.0f * pi / u[0], qa = 2.0f * pi / u[1];
    const float r2 = 1.0f - (std::cos(pa) - 1.0f) / (std::cos(pa) + std::cos(qa));
    o[0] = pa; o[1] = r2 > 0.0f ? 1.0f / std::sqrt(r2) : 1.0f;
}
void derive_blur_linear(const float* u, float* o) { o[0] = std::cos(u[1]); o[1] = std::sin(u[1]); }   // circle_blur.rs
void derive_shredrad(const float* u, float* o) {                // misc_extras4.rs (init_shredrad)
    o[0] = 6.28318530717959f / (std::fabs(u[0]) < 1e-6f ? 1e-6f : u[0]);
}
void derive_xheart(const float* u, float* o) {                  // misc_extras4.rs (init_xheart)
    const float ang = 0.7853981633974483f + 0.39269908169872414f * u[0];
    o[0] = 6.0f + 2.0f * u[1]; o[1] = std::cos(ang); o[2] = std::sin(ang);
}
void derive_pre_bwraps(const float* u, float* o) {              // pre_phase.rs (init_pre_bwraps), post_phase.rs
    derive_bwraps(u, o);
    o[3] = u[3]; o[4] = u[4];
}
void derive_hypertile2(const float* u, float* o) { derive_hypertile1(u, o); }   // hypertile.rs (init_hypertile2)
void derive_glynnSim1(const float* u, float* o) {               // glynn.rs (init_glynnSim1)
    const float a = 3.14159265358979f * u[2] / 180.0f;
    o[0] = u[0] * std::cos(a); o[1] = u[0] * std::sin(a); o[2] = std::fabs(u[4]);
}
void derive_glynnSim2(const float* u, float* o) {               // glynn.rs (init_glynnSim2)
    const float pi180 = (float)(3.14159265358979 / 180.0);      // folded in double, as the shader's constant expression
    const float p10 = pi180 * u[4], p20 = pi180 * u[5];
    o[0] = p10; o[1] = u[1] * (2.0f * u[0] + u[1]) / std::max(u[0] + u[1], 1e-30f);
    o[2] = p20 - p10; o[3] = std::fabs(u[3]); o[4] = u[0] + u[1];
}
void derive_glynnSim3(const float* u, float* o) {               // glynn.rs (init_glynnSim3)
    const float r1 = u[0] + u[1], s1 = r1 == 0.0f ? 1e-30f : r1, r2 = (u[0] * u[0]) / s1;
    o[0] = r1; o[1] = r2; o[2] = r1 / std::max(r1 + r2, 1e-30f); o[3] = std::fabs(u[3]);
}
void derive_target_sp(const float* u, float* o) {               // radial_extras.rs (init_target_sp)
    const float pi = 3.14159265358979f, rota = pi * u[0];
    o[0] = 0.5f * u[2]; o[1] = rota; o[2] = -pi + rota;
}
void derive_starblur(const float* u, float* o) {                // blur_extras.rs (init_starblur)
    const float pw = std::max(u[0], 1.0f), a0 = 3.14159265358979f / pw;
    const float len = std::sqrt(std::max(1.0f + u[1] * u[1] - 2.0f * u[1] * std::cos(a0), 1e-30f));
    o[0] = std::asin(std::sin(a0) * u[1] / len); o[1] = len;
}
void derive_vogel(const float* u, float* o) {                   // parametric_curves.rs (init_vogel)
    (void)u;
    const float phi = 1.618033988749895f;
    o[0] = 6.28318530717959f / (phi * phi);
}
void derive_cpow3(const float* u, float* o) {                   // heavy_init.rs (init_cpow3)
    const float sd = u[2] == 0.0f ? 1e-30f : u[2];
    const float log_d = u[1] < 0.0f ? -std::log(std::max(-u[1], 1e-30f)) : std::log(std::max(u[1], 1e-30f));
    const float pa = std::atan2(log_d * u[0], 6.28318530717959f), cpa = std::cos(pa);
    const float c = cpa * u[0] * std::cos(pa) / sd, d = cpa * u[0] * std::sin(pa) / sd;
    o[0] = 6.28318530717959f / sd; o[1] = c; o[2] = d; o[3] = c * 0.5f; o[4] = d * 0.5f;
    o[5] = d == 0.0f ? 0.0f : -0.095f * u[3] / d;
}
void derive_yin_yang(const float* u, float* o) {                // init_ports.rs (init_yin_yang)
    const float pi = 3.14159265358979f;
    o[0] = std::sin(pi * u[1]); o[1] = std::cos(pi * u[1]); o[2] = std::sin(pi * u[2]); o[3] = std::cos(pi * u[2]);
}
void derive_oscilloscope2(const float* u, float* o) {           // misc_extras3.rs (init_oscilloscope2)
    o[0] = 6.28318530717959f * u[1]; o[1] = 6.28318530717959f * u[2];
}
void derive_phoenix_julia(const float* u, float* o) {           // misc_extras3.rs (init_phoenix_julia)
    const float sp = u[0] == 0.0f ? 1e-30f : u[0];
    o[0] = u[1] / sp; o[1] = 6.28318530717959f / sp; o[2] = u[1] / sp * 0.5f;
}
void derive_pow_block(const float* u, float* o) {               // misc_extras3.rs (init_pow_block)
    float pw = u[1] * u[2] / std::max(std::fabs(u[3]), 1e-30f);
    if (std::fabs(pw) <= 1e-30f) pw = 1e-30f;
    o[0] = u[0] * 0.5f / pw; o[1] = 1.0f / std::max(std::fabs(u[1]), 1e-30f);
}
void derive_trade(const float* u, float* o) { o[0] = u[0] + u[1]; o[1] = u[2] + u[3]; }   // watchlist_misc.rs (init_trade)
void derive_checks(const float* u, float* o) { o[0] = 1.0f / (u[2] + 1e-30f); }           // apo_misc.rs (init_checks)
void derive_boarders2(const float* u, float* o) {               // boarders.rs (init_boarders2)
    const float c0 = std::max(std::fabs(u[0]), 1e-6f), cl0 = std::max(std::fabs(u[1]), 1e-6f), cr0 = std::max(std::fabs(u[2]), 1e-6f);
    o[0] = c0; o[1] = c0 * cl0; o[2] = c0 + c0 * cr0;
}
void derive_squish(const float* u, float* o) { o[0] = 1.0f / std::max(u[0], 2.0f); }   // classic_blades_misc.rs (init_squish)
void derive_eJulia(const float* u, float* o) { o[0] = u[0] < 0.0f ? -1.0f : 1.0f; }     // apo_misc9.rs (init_eJulia)
void derive_julian2(const float* u, float* o) {                 // apo_misc9.rs (init_julian2)
    const float sp = std::fabs(u[0]) < 1e-30f ? 1.0f : u[0];
    o[0] = std::fabs(sp); o[1] = u[1] / (2.0f * sp);
}
// WGSL's saturating f32 -> i32 (toward zero, clamped, NaN 0).
int32_t sat_i32f(float f) {
    if (std::isnan(f)) return 0;
    if (f <= -2147483648.0f) return INT32_MIN;
    if (f >= 2147483648.0f) return INT32_MAX;
    return (int32_t)f;
}
void derive_npolar(const float* u, float* o) {                  // apo_misc7.rs (init_npolar)
    const int p = sat_i32f(u[0]), n = sat_i32f(u[1]), nz = n == 0 ? 1 : n;
    const int ap = std::abs(p), odd = ap - (ap / 2) * 2;
    o[0] = (float)nz; o[1] = (float)odd; o[2] = (float)std::abs(nz); o[3] = 1.0f / (2.0f * (float)nz);
}
void derive_waffle(const float* u, float* o) { o[0] = std::cos(u[3]); o[1] = std::sin(u[3]); }   // apo_misc12.rs (init_waffle)
void derive_ripple(const float* u, float* o) {                  // apo_misc13.rs (init_ripple)
    const float pi = 3.14159265358979f, tp = 6.28318530717959f;
    const float al = u[2] * 0.01f, pl = u[5] * tp - pi, s = std::fabs(u[6]) < 1e-30f ? 1e-30f : u[6];
    o[0] = u[0] * 5.0f; o[1] = pl; o[2] = s; o[3] = u[1] * pl; o[4] = pl * al; o[5] = (pi - pl) * al;
}
void derive_circlecrop(const float* u, float* o) { o[0] = std::min(std::max(u[3], -1.0f), 1.0f); }   // circlecrop_*.rs (init)
void derive_minkowskope(const float* u, float* o) { o[0] = 0.5f * u[1]; o[1] = 0.5f * u[2]; }   // minkowskope_misc.rs (init)
void derive_glynnlissa(const float* u, float* o) {              // glynnlissa_misc.rs (init)
    const float pi = 3.14159265358979f, phi = u[3] * pi / 180.0f;
    o[0] = u[0] * std::cos(phi); o[1] = u[0] * std::sin(phi); o[2] = std::fabs(u[9]);
}
void derive_crop3D(const float* u, float* o) {                  // parametric_curves.rs (init_crop3D)
    o[0] = std::fmin(u[0], u[3]); o[1] = std::fmax(u[0], u[3]); o[2] = std::fmin(u[1], u[4]);
    o[3] = std::fmax(u[1], u[4]); o[4] = std::fmin(u[2], u[5]); o[5] = std::fmax(u[2], u[5]);
}
void derive_spherecrop(const float* u, float* o) { o[0] = std::min(std::max(u[4], -1.0f), 1.0f); }   // apo_misc18.rs (init)
void derive_spherical3D_wf(const float* u, float* o) { o[0] = std::fabs(u[1] - 2.0f) < 1e-6f ? 1.0f : 0.0f; }   // apo_misc20.rs
void derive_hypertile3D(const float* u, float* o) {             // hypertile.rs (init_hypertile3D)
    const float pi = 3.14159265358979f, pa = 2.0f * pi / u[0], qa = 2.0f * pi / u[1];
    const float r_alt = -(std::cos(pa) - 1.0f) / (std::cos(pa) + std::cos(qa));
    const float r = r_alt > 0.0f ? 1.0f / std::sqrt(1.0f + r_alt) : 1.0f, na = u[2] * pa;
    const float cx = r * std::cos(na), cy = r * std::sin(na), cx2 = cx * cx, cy2 = cy * cy;
    o[0] = cx; o[1] = cy; o[2] = cx2 + cy2; o[3] = 2.0f * cx; o[4] = 2.0f * cy;
    o[5] = 1.0f + cx2 - cy2; o[6] = 1.0f + cy2 - cx2; o[7] = 1.0f - cx2 - cy2;
}
void derive_hypercrop(const float* u, float* o) {               // maurer_hyper.rs (init_hypercrop)
    const float n = std::fmax(u[0], 3.0f), a0 = 3.14159265358979f / n, len = 1.0f / std::cos(a0);
    o[0] = n / 6.28318530717959f; o[1] = a0; o[2] = len; o[3] = u[1] * std::sin(a0) * len;
}
void derive_poincare3D(const float* u, float* o) {              // apo_misc14.rs (init_poincare3D)
    const float h = 1.5707963267948966f, r = u[0], cb = std::cos(u[2] * h);
    const float cx = -r * std::cos(u[1] * h) * cb, cy = r * std::sin(u[1] * h) * cb, cz = -r * std::sin(u[2] * h);
    const float cx2 = cx * cx, cy2 = cy * cy, cz2 = cz * cz;
    o[0] = cx; o[1] = cy; o[2] = cz; o[3] = cx2 + cy2 + cz2; o[4] = 2.0f * cx; o[5] = 2.0f * cy; o[6] = 2.0f * cz;
    o[7] = cx2 - cy2 - cz2 + 1.0f; o[8] = cy2 - cx2 - cz2 + 1.0f; o[9] = cz2 - cy2 - cx2 + 1.0f;
}
void derive_rosoni(const float* u, float* o) {                  // rosoni_misc.rs (init_rosoni)
    const float phi = 6.28318530717959f / std::fmax(u[0], 1.0f);
    o[0] = std::sin(phi); o[1] = std::cos(phi);
}
void derive_bwraps7(const float* u, float* o) {                 // bwraps7_misc.rs (init_bwraps7)
    if (std::fabs(u[0]) < 1e-30f) { o[0] = o[1] = o[2] = 0.0f; return; }
    const float radius = 0.5f * (u[0] / (1.0f + u[1] * u[1])), g2 = u[2] * u[2] + 1e-6f;
    float mb = g2 * radius;
    mb = mb > 2.0f ? 1.0f : mb * (1.0f / ((mb * mb) * 0.25f + 1.0f));
    o[0] = g2; o[1] = radius * radius; o[2] = radius / std::fmax(mb, 1e-30f);
}
void derive_curl_sp(const float* u, float* o) {                 // curl_sp_misc.rs (init_curl_sp)
    const float p = std::fabs(u[0]) < 1e-30f ? 1e-6f : u[0];
    o[0] = p; o[1] = 2.0f * u[2]; o[2] = 1.0f / p; o[3] = 0.1f * u[5];
}
void derive_waves_wf(const float* u, float* o) {                // waves_wf_family.rs (init_waves2_wf, shared)
    o[0] = std::fabs(u[6]) < 1e-6f ? 1.0f : std::exp(u[6]);
    o[1] = std::fabs(u[7]) < 1e-6f ? 1.0f : std::exp(u[7]);
}
void derive_xheart_blur_wf(const float* u, float* o) {          // apo_misc18.rs (init_xheart_blur_wf)
    const float pi_4 = 0.7853981633974483f, ang = pi_4 + 0.5f * pi_4 * u[0];
    o[0] = std::sin(ang); o[1] = std::cos(ang); o[2] = 6.0f + 2.0f * u[1];
}
void derive_affine3D(const float* u, float* o) {                // affine3d_misc.rs (init_affine3D)
    const float d2r = 0.017453292519943295f;
    const bool shear = std::fabs(u[9]) + std::fabs(u[10]) + std::fabs(u[11]) + std::fabs(u[12]) + std::fabs(u[13]) + std::fabs(u[14]) > 1e-6f;
    o[0] = std::sin(u[6] * d2r); o[1] = std::cos(u[6] * d2r); o[2] = std::sin(u[7] * d2r); o[3] = std::cos(u[7] * d2r);
    o[4] = std::sin(u[8] * d2r); o[5] = std::cos(u[8] * d2r); o[6] = shear ? 1.0f : 0.0f;
}
// z and w (wz_lost_variations.rs init_z, init_w): `h` the index of hypergon.
void derive_wz(const float* u, float* o, int h) {
    o[0] = std::sqrt(1.0f + u[h + 2] * u[h + 2]); o[1] = u[h + 1]; o[2] = -u[h + 7]; o[3] = u[h + 4];
    o[4] = std::tan(u[h + 5]); o[5] = u[h + 9] * 0.25f; o[6] = -1.0f / (u[h + 10] + 1e-7f);
}
void derive_z(const float* u, float* o) { derive_wz(u, o, 0); }
void derive_w(const float* u, float* o) { derive_wz(u, o, 1); }
void derive_loonie2(const float* u, float* o) {                 // watchlist_misc.rs (init_loonie2), apo_misc13.rs (init_scry2)
    const float a = 6.28318530717959f / std::fmax(u[0], 1.0f), as = -1.5707963267948966f * u[1], ac = 1.5707963267948966f * u[2];
    o[0] = std::sin(a); o[1] = std::cos(a); o[2] = std::sin(as); o[3] = std::cos(as); o[4] = std::sin(ac); o[5] = std::cos(ac);
}
void derive_elliptic2(const float* u, float* o) { o[0] = u[10] * 0.31830988618379f; }   // erf_misc.rs (init_elliptic2)
void derive_asteria(const float* u, float* o) {                 // apo_misc7.rs (init_asteria)
    o[0] = std::sin(3.14159265358979f * u[0]); o[1] = std::cos(3.14159265358979f * u[0]);
}
void derive_bwraps2(const float* u, float* o) {                 // bwraps2_phase.rs (init_pre_bwraps2, init_post_bwraps2)
    if (std::fabs(u[0]) < 1e-30f) { o[0] = o[1] = o[2] = 0.0f; return; }
    const float radius = 0.5f * (u[0] / (1.0f + u[1] * u[1])), g2 = u[2] * u[2] / u[0] + 1e-6f;
    float mb = g2 * radius;
    mb = mb > 2.0f ? 1.0f : mb * (1.0f / ((mb * mb) * 0.25f + 1.0f));
    o[0] = g2; o[1] = radius * radius; o[2] = radius / std::fmax(mb, 1e-30f);
}
void derive_post_rblur(const float* u, float* o) { o[0] = 2.0f * u[0]; }   // post_rblur_misc.rs (init_post_rblur)
void derive_cpow3_wf(const float* u, float* o) {                // apo_misc22.rs (init_cpow3_wf)
    const float pi = 3.14159265358979f, two_pi = 6.28318530717959f;
    const float div = std::fabs(u[2]) < 1e-30f ? 1e-30f : u[2], spr = std::fabs(u[3]) < 1e-30f ? 1e-30f : u[3];
    const float c = u[0] * std::cos(pi * 0.5f * u[1]) / div, d = u[0] * std::sin(pi * 0.5f * u[1]) / div;
    o[0] = c; o[1] = d; o[2] = c * 0.5f; o[3] = d * 0.5f; o[4] = two_pi / div; o[5] = 0.5f / spr; o[6] = two_pi * u[3];
}
void derive_pre_rect_wf(const float* u, float* o) { o[0] = u[1] - u[0]; o[1] = u[3] - u[2]; }   // dc_misc2.rs (init_pre_rect_wf)
void derive_spliptic_bs(const float*, float* o) { o[0] = 0.6366197723675814f; }   // apo_misc14.rs (init_spliptic_bs)
void derive_pointgrid_wf(const float* u, float* o) {            // pointgrid_misc.rs (init_pointgrid_wf)
    o[0] = (u[1] - u[0]) / std::fmax(u[2], 1.0f); o[1] = (u[4] - u[3]) / std::fmax(u[5], 1.0f);
}
void derive_bubbleT3D(const float* u, float* o) {               // bubblet3d_misc.rs (init_bubbleT3D)
    const float pi = 3.14159265358979f, two_pi = 6.28318530717959f, as = std::fabs(u[0]);
    const float ratio = std::fmin(std::fmax(u[1], 0.01f), 1.99f);
    float s = 0.0f, s1 = 0.0f, s2 = 0.0f;
    if (as > 0.5f) { s = pi / as; s2 = 2.0f * s; s1 = ratio * s; }
    float ah = u[2];
    if (u[4] > 0.5f) ah = std::fmin(std::fabs(ah), 179.9f);
    const float inv_hole = ah < 0.0f ? 1.0f : 0.0f;
    float ae = std::fabs(ah);
    ae = inv_hole > 0.5f ? (ae / 360.0f * two_pi) * 0.5f : pi - (ae / 360.0f * two_pi) * 0.5f;
    o[0] = pi - ae; o[1] = s; o[2] = s1; o[3] = s2; o[4] = u[0] < 0.0f ? 1.0f : 0.0f; o[5] = inv_hole; o[6] = ae;
}
// hypertile3D1, hypertile3D2 (hypertile.rs init_hypertile3D1, 2): the tile
// angle 2 pi / p and the tile centre's distance r.
void ffb_hypertile3_r(const float* u, float& pa, float& r) {
    const float pi = 3.14159265358979f, qa = 2.0f * pi / u[1];
    pa = 2.0f * pi / u[0];
    const float r_alt = -(std::cos(pa) - 1.0f) / (std::cos(pa) + std::cos(qa));
    r = r_alt > 0.0f ? 1.0f / std::sqrt(1.0f + r_alt) : 1.0f;
}
void derive_hypertile3D1(const float* u, float* o) {
    float pa, r;
    ffb_hypertile3_r(u, pa, r);
    o[0] = pa; o[1] = r; o[2] = r * r; o[3] = 1.0f - r * r;
}
void derive_hypertile3D2(const float* u, float* o) {
    float pa, r;
    ffb_hypertile3_r(u, pa, r);
    const float cx2 = r * r;
    o[0] = pa; o[1] = r; o[2] = cx2; o[3] = 2.0f * r; o[4] = 1.0f + cx2; o[5] = 1.0f - cx2; o[6] = 1.0f - cx2;
}
void derive_julian3Dx(const float* u, float* o) {               // apo_misc15.rs (init_julian3Dx)
    const float p = std::fabs(u[0]) < 1e-30f ? 1.0f : u[0];
    o[0] = std::fabs(p); o[1] = (u[1] / p - 1.0f) * 0.5f;
}
void derive_waves2b(const float* u, float* o) { o[0] = u[4] - u[5]; o[1] = u[6] - u[7]; }   // waves2b_misc.rs (init_waves2b)
void derive_log_db(const float* u, float* o) {                  // exp_log.rs (init_log_db)
    o[0] = u[0] <= 1e-20f ? 0.5f : 0.5f / std::log(std::fmax(2.71828182845905f * u[0], 1e-20f));
    o[1] = u[1] <= 1e-20f ? 3.14159265358979f : 3.14159265358979f * u[1];
}
void derive_juliaq(const float* u, float* o) {                  // numbered.rs (init_juliaq)
    const float power = std::fmax(u[0], 1.0f), ip = u[1] / power;
    o[0] = ip; o[1] = 6.28318530717959f / power; o[2] = 0.5f * ip;
}
void derive_julia3Dq(const float* u, float* o) {                // numbered.rs (init_julia3Dq)
    const float power = std::fmax(u[0], 1.0f), ip = u[1] / power;
    o[0] = ip; o[1] = 6.28318530717959f / power; o[2] = 0.5f * ip - 0.5f; o[3] = std::fabs(ip);
}
void derive_juliac(const float* u, float* o) { o[0] = 1.0f / (u[0] + 1e-30f); o[1] = u[1] / 100.0f; }   // numbered.rs (init_juliac)
void derive_cpow2(const float* u, float* o) {                   // heavy_init.rs (init_cpow2)
    const float sd = u[2] == 0.0f ? 1e-30f : u[2], range = std::fmax(u[3], 1.0f);
    const float c = u[0] * std::cos(1.5707963267948966f * u[1]) / sd, d = u[0] * std::sin(1.5707963267948966f * u[1]) / sd;
    o[0] = 6.28318530717959f / sd; o[1] = c; o[2] = d; o[3] = c * 0.5f; o[4] = d * 0.5f; o[5] = 0.5f / range;
    o[6] = 6.28318530717959f * range;
}
void derive_post_juliaq(const float* u, float* o) {             // pre_post_bridges.rs (init_post_juliaq)
    const float sp = u[0] == 0.0f ? 1e-30f : u[0];
    o[0] = 0.5f * u[1] / sp; o[1] = u[1] / sp; o[2] = 6.28318530717959f / sp;
}
void derive_post_julia3Dq(const float* u, float* o) {           // pre_post_bridges.rs (init_post_julia3Dq)
    const float sp = u[0] == 0.0f ? 1e-30f : u[0], ip = u[1] / sp;
    o[0] = ip; o[1] = std::fabs(ip); o[2] = 0.5f * ip - 0.5f; o[3] = 6.28318530717959f / sp;
}
// cut_fractal's constant c and cut_snowflake's starting depth, functions of
// the time parameter alone (cut_simple.rs), taken once on the host.
void derive_cut_fractal(const float* u, float* o) {
    o[0] = std::cos(u[2] + 1.5f) * 0.15f - 0.25f; o[1] = std::sin(u[2] + 1.8f) * 0.15f - 0.25f;
}
void derive_cut_snowflake(const float* u, float* o) { o[0] = std::sin(u[2] * 0.4f) * 0.5f - 0.5f; }
}  // namespace

// The variations this build carries, in the reference's registry order
// (ALL_VARIATIONS, src/variations/defs/mod.rs:446; `id` is the position
// there).  Bodies live in ffb_device.cuh; parameters, their defaults, the
// draws each body takes and the derived values from the defs
// (src/variations/defs/*.rs, cited at each body).
#define NP {nullptr}
#define ND {0}
static const VarDef kRegistry[] = {
    {"linear", 0, 0, 0, NP, ND, "v_linear", VF_JAC, 0, nullptr},
    {"sinusoidal", 1, 0, 0, NP, ND, "v_sinusoidal", VF_JAC, 0, nullptr},
    {"spherical", 2, 0, 0, NP, ND, "v_spherical", VF_JAC, 0, nullptr},
    {"swirl", 3, 0, 0, NP, ND, "v_swirl", VF_JAC, 0, nullptr},
    {"horseshoe", 4, 0, 0, NP, ND, "v_horseshoe", VF_JAC, 0, nullptr},
    {"polar", 5, 0, 0, NP, ND, "v_polar", VF_JAC, 0, nullptr},
    {"handkerchief", 6, 0, 0, NP, ND, "v_handkerchief", 0, 0, nullptr},
    {"heart", 7, 0, 0, NP, ND, "v_heart", 0, 0, nullptr},
    {"disc", 8, 0, 0, NP, ND, "v_disc", VF_JAC, 0, nullptr},
    {"spiral", 9, 0, 0, NP, ND, "v_spiral", 0, 0, nullptr},
    {"hyperbolic", 10, 0, 0, NP, ND, "v_hyperbolic", 0, 0, nullptr},
    {"diamond", 11, 0, 0, NP, ND, "v_diamond", 0, 0, nullptr},
    {"ex", 12, 0, 0, NP, ND, "v_ex", VF_JAC, 0, nullptr},
    {"julia", 13, 1, 0, NP, ND, "v_julia", VF_JAC, 0, nullptr},
    {"bent", 14, 0, 0, NP, ND, "v_bent", 0, 0, nullptr},
    {"waves", 15, 0, 0, NP, ND, "v_waves", VF_XF, 0, nullptr},
    {"zcone", 16, 0, 0, NP, ND, "v_zcone", 0, 0, nullptr},
    {"flatten", 17, 0, 0, NP, ND, "v_flatten", VF_POST, 0, nullptr},
    {"hemisphere", 18, 0, 0, NP, ND, "v_hemisphere", 0, 0, nullptr},
    {"pre_rotate_x", 19, 0, 0, NP, ND, "v_pre_rotate_x", VF_PRE, 0, nullptr},
    {"pre_rotate_y", 20, 0, 0, NP, ND, "v_pre_rotate_y", VF_PRE, 0, nullptr},
    {"post_rotate_x", 21, 0, 0, NP, ND, "v_post_rotate_x", VF_POST, 0, nullptr},
    {"post_rotate_y", 22, 0, 0, NP, ND, "v_post_rotate_y", VF_POST, 0, nullptr},
    {"zscale", 23, 0, 0, NP, ND, "v_zscale", 0, 0, nullptr},
    {"julian", 24, 1, 2, {"power", "dist"}, {2.0f, 1.0f}, "v_julian", 0, 1, derive_julian},
    {"blob", 25, 0, 3, {"high", "low", "waves"}, {1.0f, 1.0f, 6.0f}, "v_blob", 0, 0, nullptr},
    {"eyefish", 26, 0, 0, NP, ND, "v_eyefish", 0, 0, nullptr},
    {"bubble", 27, 0, 0, NP, ND, "v_bubble", VF_JAC, 0, nullptr},
    {"cylinder", 28, 0, 0, NP, ND, "v_cylinder", VF_JAC, 0, nullptr},
    {"noise", 29, 2, 0, NP, ND, "v_noise", 0, 0, nullptr},
    {"blur", 30, 2, 0, NP, ND, "v_blur", 0, 0, nullptr},
    {"gaussian_blur", 31, 5, 0, NP, ND, "v_gaussian_blur", 0, 0, nullptr},
    {"polar2", 32, 0, 0, NP, ND, "v_polar2", 0, 0, nullptr},
    {"cross", 33, 0, 0, NP, ND, "v_cross", 0, 0, nullptr},
    {"loonie", 34, 0, 0, NP, ND, "v_loonie", 0, 0, nullptr},
    {"scry", 35, 0, 0, NP, ND, "v_scry", 0, 0, nullptr},
    {"scry_3D", 36, 0, 0, NP, ND, "v_scry_3D", VF_W, 0, nullptr},
    {"foci", 37, 0, 0, NP, ND, "v_foci", 0, 0, nullptr},
    {"elliptic", 38, 0, 0, NP, ND, "v_elliptic", 0, 0, nullptr},
    {"waves2", 39, 0, 6, {"freqx", "scalex", "freqy", "scaley", "freqz", "scalez"}, {2.0f, 1.0f, 2.0f, 1.0f, 0.0f, 0.0f}, "v_waves2", 0, 0, nullptr},
    {"log", 40, 0, 1, {"base"}, {2.718281828f}, "v_log", 0, 1, derive_log},
    {"escher", 41, 0, 1, {"beta"}, {0.0f}, "v_escher", 0, 2, derive_escher},
    {"bipolar", 42, 0, 1, {"shift"}, {0.0f}, "v_bipolar", 0, 0, nullptr},
    {"lazysusan", 43, 0, 5, {"spin", "space", "twist", "x", "y"}, {0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, "v_lazysusan", 0, 0, nullptr},
    {"rings2", 44, 0, 1, {"val"}, {1.0f}, "v_rings2", 0, 0, nullptr},
    {"fan2", 45, 0, 2, {"x", "y"}, {1.0f, 0.0f}, "v_fan2", 0, 0, nullptr},
    {"pdj", 46, 0, 4, {"a", "b", "c", "d"}, {0.0f, 0.0f, 0.0f, 0.0f}, "v_pdj", 0, 0, nullptr},
    {"curl", 47, 0, 2, {"c1", "c2"}, {1.0f, 0.0f}, "v_curl", VF_JAC, 0, nullptr},
    {"rectangles", 48, 0, 2, {"x", "y"}, {1.0f, 1.0f}, "v_rectangles", 0, 0, nullptr},
    {"splits", 49, 0, 6, {"x", "y", "lshear", "rshear", "ushear", "dshear"}, {0.4f, 0.4f, 0.0f, 0.0f, 0.0f, 0.0f},
     "v_splits", 0, 0, nullptr},
    {"ngon", 50, 0, 4, {"sides", "power", "circle", "corners"}, {5.0f, 3.0f, 1.0f, 2.0f}, "v_ngon", 0, 0, nullptr},
    {"auger", 51, 0, 4, {"freq", "weight", "scale", "sym"}, {1.0f, 0.5f, 0.5f, 0.0f}, "v_auger", 0, 0, nullptr},
    {"zblur", 52, 0, 0, NP, ND, "v_zblur", 0, 0, nullptr},
    {"blur3D", 53, 6, 0, NP, ND, "v_blur3D", 0, 0, nullptr},
    {"pre_blur", 54, 7, 0, NP, ND, "v_pre_blur", VF_PRE | VF_W, 0, nullptr},
    {"pre_zscale", 55, 0, 0, NP, ND, "v_pre_zscale", VF_PRE, 0, nullptr},
    {"pre_ztranslate", 56, 0, 0, NP, ND, "v_pre_ztranslate", VF_PRE, 0, nullptr},
    {"pre_spherical", 57, 0, 0, NP, ND, "v_pre_spherical", VF_PRE, 0, nullptr},
    {"pre_sinusoidal", 58, 0, 0, NP, ND, "v_pre_sinusoidal", VF_PRE | VF_W, 0, nullptr},
    {"pre_disc", 59, 0, 0, NP, ND, "v_pre_disc", VF_PRE | VF_W, 0, nullptr},
    {"pre_bwraps", 60, 0, 5, {"cellsize", "space", "gain", "inner_twist", "outer_twist"}, {1.0f, 0.0f, 1.0f, 0.0f, 0.0f}, "v_pre_bwraps", VF_PRE, 5, derive_pre_bwraps},
    {"pre_crop", 61, 2, 6, {"left", "top", "right", "bottom", "scatter_area", "zero"}, {-1.0f, -1.0f, 1.0f, 1.0f, 0.0f, 0.0f}, "v_pre_crop", VF_PRE, 0, nullptr},
    {"pre_falloff2", 62, 3, 11, {"scatter", "mindist", "mul_x", "mul_y", "mul_z", "mul_c", "x0", "y0", "z0", "invert", "type"}, {1.0f, 0.5f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, "v_pre_falloff2", VF_PRE, 0, nullptr},
    {"ztranslate", 63, 0, 0, NP, ND, "v_ztranslate", 0, 0, nullptr},
    {"julia3D", 64, 1, 1, {"power"}, {2.0f}, "v_julia3D", 0, 0, nullptr},
    {"falloff2", 65, 2, 11, {"scatter", "mindist", "mul_x", "mul_y", "mul_z", "mul_c", "x0", "y0", "z0", "invert", "type"}, {1.0f, 0.5f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, "v_falloff2", 0, 0, nullptr},
    {"wedge", 66, 0, 4, {"angle", "hole", "count", "swirl"}, {90.0f, 0.0f, 2.0f, 0.0f}, "v_wedge", 0, 2, derive_wedge},
    {"epispiral", 67, 1, 3, {"n", "thickness", "holes"}, {6.0f, 0.0f, 1.0f}, "v_epispiral", 0, 0, nullptr},
    {"bwraps", 68, 0, 5, {"cellsize", "space", "gain", "inner_twist", "outer_twist"}, {1.0f, 0.0f, 1.0f, 0.0f, 0.0f}, "v_bwraps", 0, 3, derive_bwraps},
    {"juliascope", 69, 1, 2, {"power", "dist"}, {2.0f, 1.0f}, "v_juliascope", 0, 0, nullptr},
    {"julia3Dz", 71, 0, 1, {"power"}, {2.0f}, "v_julia3Dz", 0, 0, nullptr},
    {"curl3D", 72, 0, 3, {"cx", "cy", "cz"}, {0.0f, 0.0f, 0.0f}, "v_curl3D", 0, 0, nullptr},
    {"radial_blur", 73, 4, 1, {"angle"}, {0.0f}, "v_radial_blur", VF_W, 2, derive_radial_blur},
    {"blur_circle", 74, 2, 0, NP, ND, "v_blur_circle", 0, 0, nullptr},
    {"blur_zoom", 75, 1, 3, {"length", "x", "y"}, {0.0f, 0.0f, 0.0f}, "v_blur_zoom", 0, 0, nullptr},
    {"blur_pixelize", 76, 2, 2, {"size", "scale"}, {0.1f, 1.0f}, "v_blur_pixelize", 0, 0, nullptr},
    {"separation", 77, 0, 4, {"x", "y", "xinside", "yinside"}, {1.0f, 1.0f, 0.0f, 0.0f}, "v_separation", 0, 0, nullptr},
    {"mobius", 78, 0, 8, {"re_a", "im_a", "re_b", "im_b", "re_c", "im_c", "re_d", "im_d"}, {0.1f, 0.2f, 0.2f, -0.12f, -0.15f, -0.15f, 0.21f, 0.1f}, "v_mobius", 0, 0, nullptr},
    {"crop", 79, 2, 6, {"left", "top", "right", "bottom", "scatter_area", "zero"}, {-1.0f, -1.0f, 1.0f, 1.0f, 0.0f, 0.0f}, "v_crop", VF_REPLACE, 0, nullptr},
    {"post_bwraps", 80, 0, 5, {"cellsize", "space", "gain", "inner_twist", "outer_twist"}, {1.0f, 0.0f, 1.0f, 0.0f, 0.0f}, "v_post_bwraps", VF_POST, 5, derive_pre_bwraps},
    {"post_crop", 81, 2, 6, {"left", "top", "right", "bottom", "scatter_area", "zero"}, {-1.0f, -1.0f, 1.0f, 1.0f, 0.0f, 0.0f}, "v_post_crop", VF_POST, 0, nullptr},
    {"post_falloff2", 82, 3, 11, {"scatter", "mindist", "mul_x", "mul_y", "mul_z", "mul_c", "x0", "y0", "z0", "invert", "type"}, {1.0f, 0.5f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, "v_post_falloff2", VF_POST, 0, nullptr},
    {"post_curl", 83, 0, 2, {"c1", "c2"}, {0.0f, 0.0f}, "v_post_curl", VF_POST, 0, nullptr},
    {"post_curl3D", 84, 0, 3, {"cx", "cy", "cz"}, {0.0f, 0.0f, 0.0f}, "v_post_curl3D", VF_POST, 0, nullptr},
    {"cpow", 85, 1, 3, {"r", "i", "power"}, {1.0f, 0.1f, 1.5f}, "v_cpow", 0, 3, derive_cpow},
    {"acoth", 86, 0, 0, NP, ND, "v_acoth", 0, 0, nullptr},
    {"acosh", 87, 1, 0, NP, ND, "v_acosh", 0, 0, nullptr},
    {"acosech", 88, 1, 0, NP, ND, "v_acosech", 0, 0, nullptr},
    {"arcsech", 89, 0, 0, NP, ND, "v_arcsech", 0, 0, nullptr},
    {"arcsech2", 90, 0, 0, NP, ND, "v_arcsech2", 0, 0, nullptr},
    {"arcsinh", 91, 0, 0, NP, ND, "v_arcsinh", 0, 0, nullptr},
    {"arctanh", 92, 0, 0, NP, ND, "v_arctanh", 0, 0, nullptr},
    {"sin", 93, 0, 0, NP, ND, "v_sin", 0, 0, nullptr},
    {"cos", 94, 0, 0, NP, ND, "v_cos", 0, 0, nullptr},
    {"tan", 95, 0, 0, NP, ND, "v_tan", 0, 0, nullptr},
    {"sec", 96, 0, 0, NP, ND, "v_sec", 0, 0, nullptr},
    {"csc", 97, 0, 0, NP, ND, "v_csc", 0, 0, nullptr},
    {"cot", 98, 0, 0, NP, ND, "v_cot", 0, 0, nullptr},
    {"sinh", 99, 0, 0, NP, ND, "v_sinh", 0, 0, nullptr},
    {"cosh", 100, 0, 0, NP, ND, "v_cosh", 0, 0, nullptr},
    {"tanh", 101, 0, 0, NP, ND, "v_tanh", 0, 0, nullptr},
    {"coth", 102, 0, 0, NP, ND, "v_coth", 0, 0, nullptr},
    {"sech", 103, 0, 0, NP, ND, "v_sech", 0, 0, nullptr},
    {"csch", 104, 0, 0, NP, ND, "v_csch", 0, 0, nullptr},
    {"sinq", 105, 0, 0, NP, ND, "v_sinq", 0, 0, nullptr},
    {"cosq", 106, 0, 0, NP, ND, "v_cosq", 0, 0, nullptr},
    {"tanq", 107, 0, 0, NP, ND, "v_tanq", 0, 0, nullptr},
    {"cotq", 108, 0, 0, NP, ND, "v_cotq", 0, 0, nullptr},
    {"secq", 109, 0, 0, NP, ND, "v_secq", 0, 0, nullptr},
    {"cscq", 110, 0, 0, NP, ND, "v_cscq", 0, 0, nullptr},
    {"sinhq", 111, 0, 0, NP, ND, "v_sinhq", 0, 0, nullptr},
    {"coshq", 112, 0, 0, NP, ND, "v_coshq", 0, 0, nullptr},
    {"tanhq", 113, 0, 0, NP, ND, "v_tanhq", 0, 0, nullptr},
    {"cothq", 114, 0, 0, NP, ND, "v_cothq", 0, 0, nullptr},
    {"sechq", 115, 0, 0, NP, ND, "v_sechq", 0, 0, nullptr},
    {"cschq", 116, 0, 0, NP, ND, "v_cschq", 0, 0, nullptr},
    {"sqrt_acoth", 117, 1, 0, NP, ND, "v_sqrt_acoth", 0, 0, nullptr},
    {"sqrt_acosh", 118, 1, 0, NP, ND, "v_sqrt_acosh", 0, 0, nullptr},
    {"sqrt_acosech", 119, 1, 0, NP, ND, "v_sqrt_acosech", 0, 0, nullptr},
    {"sqrt_asech", 120, 1, 0, NP, ND, "v_sqrt_asech", 0, 0, nullptr},
    {"sqrt_asinh", 121, 1, 0, NP, ND, "v_sqrt_asinh", 0, 0, nullptr},
    {"sqrt_atanh", 122, 1, 0, NP, ND, "v_sqrt_atanh", 0, 0, nullptr},
    {"sin2_bs", 123, 0, 4, {"x1", "x2", "y1", "y2"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_sin2_bs", 0, 0, nullptr},
    {"cos2_bs", 124, 0, 4, {"x1", "x2", "y1", "y2"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_cos2_bs", 0, 0, nullptr},
    {"tan2_bs", 125, 0, 4, {"x1", "x2", "y1", "y2"}, {2.0f, 2.0f, 2.0f, 2.0f}, "v_tan2_bs", 0, 0, nullptr},
    {"sec2_bs", 126, 0, 4, {"x1", "x2", "y1", "y2"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_sec2_bs", 0, 0, nullptr},
    {"csc2_bs", 127, 0, 4, {"x1", "x2", "y1", "y2"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_csc2_bs", 0, 0, nullptr},
    {"cot2_bs", 128, 0, 4, {"x1", "x2", "y1", "y2"}, {2.0f, 2.0f, 2.0f, 2.0f}, "v_cot2_bs", 0, 0, nullptr},
    {"sinh2_bs", 129, 0, 4, {"x1", "x2", "y1", "y2"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_sinh2_bs", 0, 0, nullptr},
    {"cosh2_bs", 130, 0, 4, {"x1", "x2", "y1", "y2"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_cosh2_bs", 0, 0, nullptr},
    {"tanh2_bs", 131, 0, 4, {"x1", "x2", "y1", "y2"}, {2.0f, 2.0f, 2.0f, 2.0f}, "v_tanh2_bs", 0, 0, nullptr},
    {"coth2_bs", 132, 0, 4, {"x1", "x2", "y1", "y2"}, {2.0f, 2.0f, 2.0f, 2.0f}, "v_coth2_bs", 0, 0, nullptr},
    {"sech2_bs", 133, 0, 4, {"x1", "x2", "y1", "y2"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_sech2_bs", 0, 0, nullptr},
    {"csch2_bs", 134, 0, 4, {"x1", "x2", "y1", "y2"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_csch2_bs", 0, 0, nullptr},
    {"exp2_bs", 135, 0, 3, {"x1", "y1", "y2"}, {1.0f, 1.0f, 1.0f}, "v_exp2_bs", 0, 0, nullptr},
    {"exp", 136, 0, 0, NP, ND, "v_exp", 0, 0, nullptr},
    {"log_db", 137, 7, 2, {"base", "fix_period"}, {1.0f, 1.0f}, "v_log_db", 0, 2, derive_log_db},
    {"log_tile2", 138, 4, 3, {"spreadx", "spready", "spreadz"}, {2.0f, 2.0f, 0.0f}, "v_log_tile2", 0, 0, nullptr},
    {"tile_log", 139, 2, 1, {"spread"}, {1.0f}, "v_tile_log", 0, 0, nullptr},
    {"tancos", 140, 0, 0, NP, ND, "v_tancos", 0, 0, nullptr},
    {"tangent", 141, 0, 0, NP, ND, "v_tangent", 0, 0, nullptr},
    {"tangent3D", 142, 0, 0, NP, ND, "v_tangent3D", 0, 0, nullptr},
    {"secant2", 143, 0, 0, NP, ND, "v_secant2", 0, 0, nullptr},
    {"cosine", 144, 0, 0, NP, ND, "v_cosine", 0, 0, nullptr},
    {"petal", 145, 0, 0, NP, ND, "v_petal", 0, 0, nullptr},
    {"cardioid", 146, 0, 1, {"a"}, {1.0f}, "v_cardioid", 0, 0, nullptr},
    {"helix", 147, 0, 2, {"frequency", "width"}, {1.0f, 0.5f}, "v_helix", 0, 0, nullptr},
    {"helicoid", 148, 0, 1, {"frequency"}, {1.0f}, "v_helicoid", 0, 0, nullptr},
    {"parabola", 149, 2, 2, {"width", "height"}, {1.0f, 0.5f}, "v_parabola", 0, 0, nullptr},
    {"pie", 150, 3, 3, {"slices", "rotation", "thickness"}, {6.0f, 0.0f, 0.5f}, "v_pie", 0, 0, nullptr},
    {"pie3D", 151, 3, 3, {"slices", "rotation", "thickness"}, {7.0f, 0.0f, 0.5f}, "v_pie3D", 0, 0, nullptr},
    {"butterfly", 152, 0, 0, NP, ND, "v_butterfly", 0, 0, nullptr},
    {"butterfly3D", 153, 0, 0, NP, ND, "v_butterfly3D", 0, 0, nullptr},
    {"ennepers", 154, 0, 0, NP, ND, "v_ennepers", VF_REPLACE, 0, nullptr},
    {"pyramid", 155, 0, 0, NP, ND, "v_pyramid", 0, 0, nullptr},
    {"rays2", 156, 0, 0, NP, ND, "v_rays2", VF_REPLACE, 0, nullptr},
    {"rays3", 157, 0, 0, NP, ND, "v_rays3", VF_REPLACE, 0, nullptr},
    {"spiralwing", 158, 0, 0, NP, ND, "v_spiralwing", 0, 0, nullptr},
    {"whitney_umbrella", 159, 0, 0, NP, ND, "v_whitney_umbrella", 0, 0, nullptr},
    {"chrysanthemum", 160, 1, 0, NP, ND, "v_chrysanthemum", 0, 0, nullptr},
    {"cell", 161, 0, 1, {"size"}, {0.6f}, "v_cell", 0, 0, nullptr},
    {"ennepers2", 162, 0, 3, {"a", "b", "c"}, {1.0f, 0.3333f, 0.075f}, "v_ennepers2", 0, 0, nullptr},
    {"flower", 163, 1, 2, {"holes", "petals"}, {0.4f, 7.0f}, "v_flower", 0, 0, nullptr},
    {"spherical3D", 164, 0, 0, NP, ND, "v_spherical3D", 0, 0, nullptr},
    {"sinusoidal3d", 165, 0, 0, NP, ND, "v_sinusoidal3d", 0, 0, nullptr},
    {"square", 166, 2, 0, NP, ND, "v_square", 0, 0, nullptr},
    {"square3D", 167, 2, 0, NP, ND, "v_square3D", 0, 0, nullptr},
    {"disc3d", 168, 0, 1, {"pi"}, {3.14159265358979f}, "v_disc3d", 0, 0, nullptr},
    {"bubble2", 169, 0, 3, {"x", "y", "z"}, {1.0f, 1.0f, 0.0f}, "v_bubble2", 0, 0, nullptr},
    {"popcorn2", 170, 0, 3, {"x", "y", "c"}, {1.0f, 0.5f, 1.5f}, "v_popcorn2", 0, 0, nullptr},
    {"splits3D", 171, 0, 3, {"x", "y", "z"}, {0.1f, 0.3f, 0.2f}, "v_splits3D", 0, 0, nullptr},
    {"waves2_3D", 172, 0, 2, {"freq", "scale"}, {2.0f, 1.0f}, "v_waves2_3D", 0, 0, nullptr},
    {"juliaq", 173, 1, 2, {"power", "divisor"}, {3.0f, 2.0f}, "v_juliaq", 0, 3, derive_juliaq},
    {"julia3Dq", 174, 1, 2, {"power", "divisor"}, {3.0f, 2.0f}, "v_julia3Dq", 0, 4, derive_julia3Dq},
    {"juliac", 175, 1, 3, {"re", "im", "dist"}, {3.0f, 0.5f, 1.0f}, "v_juliac", 0, 2, derive_juliac},
    {"cpow2", 176, 3, 4, {"r", "a", "divisor", "range"}, {1.0f, 0.0f, 1.0f, 1.0f}, "v_cpow2", 0, 7, derive_cpow2},
    {"cpow3", 177, 4, 4, {"r", "d", "divisor", "spread"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_cpow3", 0, 6, derive_cpow3},
    {"disc2", 178, 0, 2, {"rot", "twist"}, {2.0f, 0.5f}, "v_disc2", 0, 3, derive_disc2},
    {"target", 179, 0, 3, {"even", "odd", "size"}, {0.0f, 0.0f, 1.0f}, "v_target", 0, 1, derive_target},
    {"yin_yang", 180, 1, 5, {"radius", "ang1", "ang2", "dual_t", "outside"}, {0.5f, 0.0f, 0.0f, 1.0f, 0.0f}, "v_yin_yang", 0, 4, derive_yin_yang},
    {"popcorn", 181, 0, 0, NP, ND, "v_popcorn", VF_XF, 0, nullptr},
    {"hypertile", 184, 0, 3, {"p", "q", "n"}, {3.0f, 7.0f, 1.0f}, "v_hypertile", 0, 2, derive_hypertile},
    {"hypertile1", 185, 1, 2, {"p", "q"}, {3.0f, 7.0f}, "v_hypertile1", 0, 2, derive_hypertile1},
    {"hypertile2", 186, 1, 2, {"p", "q"}, {3.0f, 7.0f}, "v_hypertile2", 0, 2, derive_hypertile2},
    {"hypertile3D", 187, 0, 3, {"p", "q", "n"}, {3.0f, 7.0f, 0.0f}, "v_hypertile3D", 0, 8, derive_hypertile3D},
    {"hypertile3D1", 188, 1, 2, {"p", "q"}, {3.0f, 7.0f}, "v_hypertile3D1", 0, 4, derive_hypertile3D1},
    {"hypertile3D2", 189, 1, 2, {"p", "q"}, {3.0f, 7.0f}, "v_hypertile3D2", 0, 7, derive_hypertile3D2},
    {"fan", 190, 0, 0, NP, ND, "v_fan", VF_XF, 0, nullptr},
    {"fisheye", 191, 0, 0, NP, ND, "v_fisheye", 0, 0, nullptr},
    {"gridout", 192, 0, 0, NP, ND, "v_gridout", 0, 0, nullptr},
    {"circular", 193, 1, 2, {"angle", "seed"}, {90.0f, 0.0f}, "v_circular", 0, 0, nullptr},
    {"panorama1", 194, 0, 0, NP, ND, "v_panorama1", 0, 0, nullptr},
    {"panorama2", 195, 0, 0, NP, ND, "v_panorama2", 0, 0, nullptr},
    {"mobiusN", 196, 1, 10, {"re_a", "re_b", "re_c", "re_d", "im_a", "im_b", "im_c", "im_d", "power", "dist"}, {1.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 1.0f}, "v_mobiusN", 0, 0, nullptr},
    {"mobiq", 197, 0, 16, {"qat", "qax", "qay", "qaz", "qbt", "qbx", "qby", "qbz", "qct", "qcx", "qcy", "qcz", "qdt", "qdx", "qdy", "qdz"}, {1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f}, "v_mobiq", 0, 0, nullptr},
    {"circleblur", 198, 2, 0, NP, ND, "v_circleblur", 0, 0, nullptr},
    {"circlesplit", 199, 0, 2, {"radius", "split"}, {1.0f, 0.5f}, "v_circlesplit", 0, 0, nullptr},
    {"flipcircle", 200, 0, 0, NP, ND, "v_flipcircle", VF_W, 0, nullptr},
    {"blur_linear", 201, 1, 2, {"length", "angle"}, {1.0f, 0.5f}, "v_blur_linear", 0, 2, derive_blur_linear},
    {"bipolar2", 202, 0, 9, {"shift", "a", "b", "c", "d", "e", "f1", "g1", "h"}, {0.0f, 1.0f, 2.0f, 0.5f, 1.0f, 2.0f, 0.25f, 1.0f, 1.0f}, "v_bipolar2", 0, 0, nullptr},
    {"blob3D", 203, 0, 3, {"low", "high", "waves"}, {0.3f, 1.2f, 6.0f}, "v_blob3D", 0, 0, nullptr},
    {"circular2", 204, 1, 4, {"angle", "seed", "xx", "yy"}, {90.0f, 0.0f, 12.9898f, 78.233f}, "v_circular2", 0, 0, nullptr},
    {"glynnia", 205, 1, 0, NP, ND, "v_glynnia", 0, 0, nullptr},
    {"glynnia3", 206, 1, 4, {"rscale", "dscale", "rthresh", "ythresh"}, {1.0f, 1.0f, 0.0f, 0.0f}, "v_glynnia3", 0, 0, nullptr},
    {"glynnSim1", 207, 3, 6, {"radius", "radius1", "phi1", "thickness", "pow", "contrast"}, {1.0f, 0.1f, 110.0f, 0.1f, 1.5f, 0.5f}, "v_glynnSim1", 0, 3, derive_glynnSim1},
    {"glynnSim2", 208, 3, 6, {"radius", "thickness", "contrast", "pow", "phi1", "phi2"}, {1.0f, 0.1f, 0.5f, 1.5f, 110.0f, 150.0f}, "v_glynnSim2", 0, 5, derive_glynnSim2},
    {"glynnSim3", 209, 3, 4, {"radius", "thickness", "contrast", "pow"}, {1.0f, 0.1f, 0.5f, 1.5f}, "v_glynnSim3", 0, 4, derive_glynnSim3},
    {"wedge_julia", 210, 1, 4, {"power", "dist", "count", "angle"}, {7.0f, 0.2f, 2.0f, 0.3f}, "v_wedge_julia", 0, 3, derive_wedge_julia},
    {"wedge_sph", 211, 0, 4, {"angle", "hole", "count", "swirl"}, {0.2f, 0.2f, 2.0f, 0.3f}, "v_wedge_sph", 0, 1, derive_wedge_sph},
    {"super_shape", 212, 1, 6, {"rnd", "m", "n1", "n2", "n3", "holes"}, {3.0f, 1.0f, 1.0f, 1.0f, 1.0f, 0.0f}, "v_super_shape", 0, 0, nullptr},
    {"henon", 213, 0, 3, {"a", "b", "c"}, {0.5f, 1.0f, 1.0f}, "v_henon", 0, 0, nullptr},
    {"apollony", 214, 1, 0, NP, ND, "v_apollony", 0, 0, nullptr},
    {"onion", 215, 0, 2, {"centre_x", "centre_y"}, {0.0f, 0.0f}, "v_onion", VF_W, 0, nullptr},
    {"target_sp", 216, 0, 4, {"twist", "n_of_sp", "size", "tightness"}, {0.0f, 1.0f, 1.0f, 0.5f}, "v_target_sp", VF_W, 3, derive_target_sp},
    {"loonie3", 217, 0, 0, NP, ND, "v_loonie3", VF_W, 0, nullptr},
    {"loonie_3D", 218, 0, 0, NP, ND, "v_loonie_3D", VF_W, 0, nullptr},
    {"sigmoid", 219, 0, 2, {"shiftx", "shifty"}, {1.0f, 1.0f}, "v_sigmoid", VF_W, 0, nullptr},
    {"blocky", 220, 0, 3, {"x", "y", "mp"}, {1.0f, 1.0f, 4.0f}, "v_blocky", VF_W, 0, nullptr},
    {"pre_curl", 221, 0, 2, {"c1", "c2"}, {0.0f, 0.0f}, "v_pre_curl", VF_PRE | VF_W, 0, nullptr},
    {"post_juliaq", 222, 1, 2, {"power", "divisor"}, {3.0f, 2.0f}, "v_post_juliaq", VF_POST | VF_W, 3, derive_post_juliaq},
    {"post_julia3Dq", 223, 1, 2, {"power", "divisor"}, {3.0f, 2.0f}, "v_post_julia3Dq", VF_POST | VF_W, 4, derive_post_julia3Dq},
    {"sineblur", 226, 2, 1, {"power"}, {1.0f}, "v_sineblur", 0, 0, nullptr},
    {"starblur", 227, 2, 2, {"power", "range"}, {5.0f, 0.40162283f}, "v_starblur", 0, 2, derive_starblur},
    {"r_circleblur", 228, 2, 5, {"n", "seed", "dist", "min", "max"}, {1.0f, 0.0f, 0.5f, 0.1f, 1.0f}, "v_r_circleblur", 0, 0, nullptr},
    {"boarders", 229, 1, 0, NP, ND, "v_boarders", 0, 0, nullptr},
    {"boarders2", 230, 1, 3, {"c", "left", "right"}, {0.4f, 0.65f, 0.35f}, "v_boarders2", 0, 3, derive_boarders2},
    {"pre_boarders2", 231, 1, 3, {"c", "left", "right"}, {0.4f, 0.65f, 0.35f}, "v_pre_boarders2", VF_PRE | VF_W, 3, derive_boarders2},
    {"splitbrdr", 232, 1, 4, {"x", "y", "px", "py"}, {0.25f, 0.25f, 0.0f, 0.0f}, "v_splitbrdr", VF_W, 0, nullptr},
    {"kaleidoscope", 233, 0, 5, {"pull", "rotate", "line_up", "x", "y"}, {0.0f, 1.0f, 1.0f, 0.0f, 0.0f}, "v_kaleidoscope", VF_W, 0, nullptr},
    {"taurus", 234, 0, 4, {"r", "n", "inv", "sor"}, {3.0f, 5.0f, 1.5f, 1.0f}, "v_taurus", 0, 0, nullptr},
    {"hole2", 235, 0, 6, {"a", "b", "c", "d", "inside", "shape"}, {1.0f, 2.0f, 1.0f, 1.0f, 0.0f, 0.0f}, "v_hole2", 0, 0, nullptr},
    {"spirograph", 236, 2, 9, {"a", "b", "d", "c1", "c2", "tmin", "tmax", "ymin", "ymax"}, {3.0f, 2.0f, 0.0f, 0.0f, 0.0f, -1.0f, 1.0f, -1.0f, 1.0f}, "v_spirograph", 0, 0, nullptr},
    {"lissajous", 237, 2, 7, {"tmin", "tmax", "a", "b", "c", "d", "e"}, {-3.14159265f, 3.14159265f, 3.0f, 2.0f, 0.0f, 0.0f, 0.0f}, "v_lissajous", 0, 0, nullptr},
    {"vogel", 238, 1, 2, {"n", "scale"}, {20.0f, 1.0f}, "v_vogel", 0, 1, derive_vogel},
    {"crop3D", 239, 2, 8, {"left", "top", "floor", "right", "bottom", "ceiling", "scatter_area", "zero"}, {-1.0f, -1.0f, -1.0f, 1.0f, 1.0f, 1.0f, 0.0f, 0.0f}, "v_crop3D", VF_REPLACE, 6, derive_crop3D},
    {"bsplit", 240, 0, 2, {"x", "y"}, {0.0f, 0.0f}, "v_bsplit", VF_HIDE, 0, nullptr},
    {"cylinder2", 241, 0, 0, NP, ND, "v_cylinder2", 0, 0, nullptr},
    {"eclipse", 242, 0, 1, {"shift"}, {0.0f}, "v_eclipse", VF_W, 0, nullptr},
    {"lozi", 243, 0, 3, {"a", "b", "c"}, {0.5f, 1.0f, 1.0f}, "v_lozi", 0, 0, nullptr},
    {"pulse", 244, 0, 4, {"freqx", "freqy", "scalex", "scaley"}, {2.0f, 2.0f, 1.0f, 1.0f}, "v_pulse", 0, 0, nullptr},
    {"hypershift", 245, 0, 2, {"shift", "stretch"}, {2.0f, 1.0f}, "v_hypershift", VF_W, 0, nullptr},
    {"hypercrop", 247, 0, 3, {"n", "rad", "zero"}, {4.0f, 1.0f, 0.0f}, "v_hypercrop", 0, 4, derive_hypercrop},
    {"split", 248, 0, 2, {"xsize", "ysize"}, {0.4f, 0.6f}, "v_split", 0, 0, nullptr},
    {"squirrel", 249, 0, 2, {"a", "b"}, {1.0f, 1.0f}, "v_squirrel", VF_REPLACE, 0, nullptr},
    {"stripes", 250, 0, 2, {"space", "warp"}, {0.2f, 0.6f}, "v_stripes", 0, 0, nullptr},
    {"shift", 251, 0, 3, {"shift_x", "shift_y", "angle"}, {0.0f, 0.0f, 0.0f}, "v_shift", 0, 2, derive_shift},
    {"pressure_wave", 252, 0, 2, {"x_freq", "y_freq"}, {1.0f, 1.0f}, "v_pressure_wave", 0, 4, derive_pressure_wave},
    {"sphericalN", 253, 1, 2, {"power", "dist"}, {1.0f, 1.0f}, "v_sphericalN", 0, 0, nullptr},
    {"spligon", 254, 0, 2, {"sides", "i"}, {3.0f, 1.0f}, "v_spligon", 0, 3, derive_spligon},
    {"tile_hlp", 255, 1, 1, {"width"}, {1.0f}, "v_tile_hlp", VF_W, 0, nullptr},
    {"ho", 256, 0, 3, {"xpow", "ypow", "zpow"}, {3.0f, 3.0f, 3.0f}, "v_ho", 0, 0, nullptr},
    {"chunk", 257, 0, 7, {"a", "b", "c", "d", "e", "f", "mode"}, {1.0f, 0.0f, 1.0f, 0.0f, 0.0f, -1.0f, 0.0f}, "v_chunk", VF_W, 0, nullptr},
    {"pTransform", 258, 0, 5, {"rotate", "power", "move", "split", "use_log"}, {0.0f, 1.0f, 0.0f, 0.0f, 1.0f}, "v_pTransform", 0, 0, nullptr},
    {"rational3", 259, 0, 8, {"a", "b", "c", "d", "e", "f", "g", "h"}, {0.5f, 0.0f, 0.0f, 1.0f, 0.0f, 1.0f, 0.0f, 1.0f}, "v_rational3", 0, 0, nullptr},
    {"tile_reverse", 260, 1, 3, {"space", "reversal", "vertical"}, {1.0f, 1.0f, 0.0f}, "v_tile_reverse", VF_REPLACE, 0, nullptr},
    {"ortho", 261, 0, 2, {"in_p", "out_p"}, {0.0f, 0.0f}, "v_ortho", 0, 0, nullptr},
    {"bCollide", 262, 0, 2, {"num", "a"}, {1.0f, 0.0f}, "v_bCollide", 0, 0, nullptr},
    {"bMod", 263, 0, 2, {"radius", "distance"}, {1.0f, 0.0f}, "v_bMod", 0, 0, nullptr},
    {"bSwirl", 264, 0, 2, {"in_p", "out_p"}, {0.0f, 0.0f}, "v_bSwirl", 0, 0, nullptr},
    {"barycentroid", 265, 0, 4, {"a", "b", "c", "d"}, {1.0f, 0.0f, 0.0f, 1.0f}, "v_barycentroid", 0, 0, nullptr},
    {"eCollide", 266, 0, 2, {"num", "a"}, {1.0f, 0.0f}, "v_eCollide", 0, 0, nullptr},
    {"eMod", 267, 0, 2, {"radius", "distance"}, {1.0f, 0.0f}, "v_eMod", 0, 0, nullptr},
    {"eSwirl", 268, 0, 2, {"in_p", "out_p"}, {1.2f, 0.2f}, "v_eSwirl", 0, 0, nullptr},
    {"eScale", 269, 0, 2, {"scale", "angle"}, {1.0f, 0.0f}, "v_eScale", 0, 0, nullptr},
    {"ePush", 270, 0, 3, {"push", "dist", "rotate"}, {0.0f, 1.0f, 0.0f}, "v_ePush", 0, 0, nullptr},
    {"eRotate", 271, 0, 1, {"rotate"}, {0.0f}, "v_eRotate", 0, 0, nullptr},
    {"corners", 272, 0, 9, {"xwidth", "ywidth", "multx", "multy", "xpower", "ypower", "xypower", "logmode", "log_base"}, {1.0f, 1.0f, 1.0f, 1.0f, 0.75f, 0.75f, 0.0f, 0.0f, 2.71828f}, "v_corners", VF_W, 0, nullptr},
    {"modulus", 273, 0, 2, {"x", "y"}, {0.2f, 0.5f}, "v_modulus", 0, 2, derive_modulus},
    {"octagon", 274, 0, 3, {"x", "y", "z"}, {0.0f, 0.0f, 0.0f}, "v_octagon", 0, 0, nullptr},
    {"circus", 275, 0, 1, {"scale"}, {1.0f}, "v_circus", 0, 1, derive_circus},
    {"circlize", 276, 0, 1, {"hole"}, {0.4f}, "v_circlize", VF_W, 0, nullptr},
    {"circlize2", 277, 0, 1, {"hole"}, {0.0f}, "v_circlize2", 0, 0, nullptr},
    {"atan", 278, 0, 2, {"mode", "stretch"}, {0.0f, 1.0f}, "v_atan", 0, 0, nullptr},
    {"murl", 279, 0, 2, {"c", "power"}, {0.1f, 1.0f}, "v_murl", 0, 3, derive_murl},
    {"collideoscope", 280, 0, 2, {"a", "num"}, {0.2f, 1.0f}, "v_collideoscope", 0, 0, nullptr},
    {"bent2", 281, 0, 2, {"x", "y"}, {1.0f, 1.0f}, "v_bent2", 0, 0, nullptr},
    {"mcarpet", 282, 0, 4, {"x", "y", "twist", "tilt"}, {1.0f, 1.0f, 0.0f, 0.0f}, "v_mcarpet", 0, 0, nullptr},
    {"linearT3D", 283, 0, 3, {"powX", "powY", "powZ"}, {1.2f, 1.2f, 1.2f}, "v_linearT3D", 0, 0, nullptr},
    {"oscilloscope", 284, 0, 4, {"separation", "frequency", "amplitude", "damping"}, {1.0f, 3.14159265f, 1.0f, 0.0f}, "v_oscilloscope", 0, 1, derive_oscilloscope},
    {"fibonacci2", 285, 0, 2, {"sc", "sc2"}, {1.0f, 1.0f}, "v_fibonacci2", 0, 0, nullptr},
    {"oscilloscope2", 286, 0, 6, {"separation", "frequencyx", "frequencyy", "amplitude", "perturbation", "damping"}, {1.0f, 3.14159265f, 3.14159265f, 1.0f, 1.0f, 0.0f}, "v_oscilloscope2", 0, 2, derive_oscilloscope2},
    {"linearT", 287, 0, 2, {"powX", "powY"}, {1.2f, 1.2f}, "v_linearT", 0, 0, nullptr},
    {"phoenix_julia", 288, 1, 4, {"power", "dist", "x_distort", "y_distort"}, {3.0f, 1.0f, -0.5f, 0.0f}, "v_phoenix_julia", 0, 3, derive_phoenix_julia},
    {"pow_block", 289, 1, 5, {"numerator", "denominator", "correctn", "correctd", "root"}, {3.0f, 2.0f, 1.0f, 1.0f, 1.0f}, "v_pow_block", 0, 2, derive_pow_block},
    {"disc3", 290, 0, 8, {"a", "b", "c", "d", "e", "f", "g", "h"}, {1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f}, "v_disc3", 0, 0, nullptr},
    {"projective", 291, 0, 9, {"a", "b", "c", "a1", "b1", "c1", "a2", "b2", "c2"}, {0.0f, 0.0f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f}, "v_projective", 0, 0, nullptr},
    {"tqmirror", 292, 0, 9, {"a", "b", "c", "d", "e", "f", "g", "h", "type"}, {1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 0.0f}, "v_tqmirror", VF_W, 0, nullptr},
    {"anamorphcyl", 296, 0, 3, {"a", "b", "k"}, {1.0f, 1.3f, 3.0f}, "v_anamorphcyl", VF_REPLACE, 0, nullptr},
    {"svf", 297, 0, 1, {"n"}, {2.0f}, "v_svf", 0, 0, nullptr},
    {"shredlin", 298, 0, 4, {"xdistance", "xwidth", "ydistance", "ywidth"}, {1.0f, 0.5f, 1.0f, 0.5f}, "v_shredlin", VF_REPLACE, 0, nullptr},
    {"shredrad", 299, 0, 2, {"n", "width"}, {4.0f, 0.5f}, "v_shredrad", 0, 1, derive_shredrad},
    {"xheart", 300, 0, 2, {"angle", "ratio"}, {0.0f, 0.0f}, "v_xheart", 0, 3, derive_xheart},
    {"stwin", 301, 0, 4, {"distort", "offset_xy", "offset_x2", "offset_y2"}, {1.0f, 0.0f, 0.0f, 0.0f}, "v_stwin", VF_W, 0, nullptr},
    {"whorl", 302, 0, 2, {"inside", "outside"}, {0.1f, 0.2f}, "v_whorl", VF_W, 0, nullptr},
    {"devil_warp", 303, 0, 6, {"a", "b", "effect", "warp", "rmin", "rmax"}, {2.0f, 1.0f, 1.0f, 0.5f, -0.24f, 100.0f}, "v_devil_warp", VF_W, 0, nullptr},
    {"trade", 304, 0, 4, {"r1", "d1", "r2", "d2"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_trade", 0, 2, derive_trade},
    {"voron", 305, 0, 5, {"k", "step", "num", "xseed", "yseed"}, {0.99f, 0.25f, 1.0f, 3.0f, 7.0f}, "v_voron", 0, 0, nullptr},
    {"squircular", 306, 0, 0, NP, ND, "v_squircular", VF_W, 0, nullptr},
    {"flux", 307, 0, 1, {"spread"}, {0.3f}, "v_flux", VF_W, 0, nullptr},
    {"rays", 308, 1, 0, NP, ND, "v_rays", VF_W, 0, nullptr},
    {"rays1", 309, 0, 0, NP, ND, "v_rays1", VF_W | VF_REPLACE, 0, nullptr},
    {"loonie2", 310, 0, 3, {"sides", "star", "circle"}, {4.0f, 0.0f, 0.0f}, "v_loonie2", VF_W, 6, derive_loonie2},
    {"fourth", 311, 0, 5, {"spin", "space", "twist", "x", "y"}, {3.14159265f, 0.0f, 0.0f, 0.0f, 0.0f}, "v_fourth", VF_W, 0, nullptr},
    {"arch", 312, 1, 0, NP, ND, "v_arch", VF_W, 0, nullptr},
    {"bi_linear", 313, 0, 0, NP, ND, "v_bi_linear", 0, 0, nullptr},
    {"blade", 314, 1, 0, NP, ND, "v_blade", VF_W, 0, nullptr},
    {"blade3D", 315, 1, 0, NP, ND, "v_blade3D", VF_W, 0, nullptr},
    {"squarize", 316, 0, 0, NP, ND, "v_squarize", 0, 0, nullptr},
    {"squish", 317, 1, 1, {"power"}, {2.0f}, "v_squish", 0, 1, derive_squish},
    {"twoface", 318, 0, 0, NP, ND, "v_twoface", VF_W, 0, nullptr},
    {"twintrian", 319, 1, 0, NP, ND, "v_twintrian", VF_W, 0, nullptr},
    {"unpolar", 320, 0, 0, NP, ND, "v_unpolar", VF_W, 0, nullptr},
    {"xerf", 321, 0, 0, NP, ND, "v_xerf", 0, 0, nullptr},
    {"inverted_julia", 322, 1, 9, {"power", "y2_mult", "a2x_mult", "a2y_mult", "a2y_add", "cos_mult", "y_mult", "center", "x2y2_add"}, {0.25f, 1.0f, 1.0f, 1.0f, 0.0f, 0.0f, 1.0f, 3.14f, 0.0f}, "v_inverted_julia", 0, 0, nullptr},
    {"idisc", 323, 0, 0, NP, ND, "v_idisc", VF_W, 0, nullptr},
    {"conic", 324, 1, 2, {"eccentricity", "holes"}, {1.0f, 0.0f}, "v_conic", VF_W, 0, nullptr},
    {"power", 325, 0, 0, NP, ND, "v_power", 0, 0, nullptr},
    {"roundspher", 326, 0, 0, NP, ND, "v_roundspher", VF_W, 0, nullptr},
    {"roundspher3D", 327, 0, 0, NP, ND, "v_roundspher3D", VF_W, 0, nullptr},
    {"checks", 330, 2, 4, {"x", "y", "size", "rnd"}, {0.5f, 0.5f, 0.5f, 0.0f}, "v_checks", 0, 1, derive_checks},
    {"cone", 331, 1, 9, {"radius1", "radius2", "size1", "size2", "ywave", "xwave", "height", "warp", "weight"}, {0.5f, 1.0f, 0.5f, 2.0f, 1.0f, 1.0f, 1.0f, 1.0f, 2.0f}, "v_cone", 0, 0, nullptr},
    {"erf", 332, 0, 0, NP, ND, "v_erf", 0, 0, nullptr},
    {"erf3D", 333, 0, 0, NP, ND, "v_erf3D", 0, 0, nullptr},
    {"d_spherical", 334, 1, 1, {"d_spher_weight"}, {0.5f}, "v_d_spherical", 0, 0, nullptr},
    {"dustpoint", 335, 2, 0, NP, ND, "v_dustpoint", 0, 0, nullptr},
    {"deltaA", 336, 0, 0, NP, ND, "v_deltaA", VF_W, 0, nullptr},
    {"edisc", 337, 0, 0, NP, ND, "v_edisc", VF_W, 0, nullptr},
    {"curve", 338, 0, 4, {"xamp", "yamp", "xlength", "ylength"}, {0.25f, 0.5f, 1.0f, 1.0f}, "v_curve", 0, 2, derive_curve},
    {"elliptic2", 339, 1, 11, {"a1", "a2", "a3", "b1", "b2", "c", "d", "e", "f", "g", "h"}, {1.0f, 1.0f, 0.0f, 2.0f, 1.0f, 0.5f, 1.0f, 0.5f, 1.0f, 1.0f, 2.0f}, "v_elliptic2", VF_W, 1, derive_elliptic2},
    {"exp2", 340, 0, 0, NP, ND, "v_exp2", 0, 0, nullptr},
    {"exponential", 341, 0, 0, NP, ND, "v_exponential", 0, 0, nullptr},
    {"flipy", 342, 0, 0, NP, ND, "v_flipy", 0, 0, nullptr},
    {"funnel", 343, 0, 1, {"effect"}, {8.0f}, "v_funnel", 0, 0, nullptr},
    {"invpolar", 344, 0, 0, NP, ND, "v_invpolar", 0, 0, nullptr},
    {"perspective", 345, 0, 2, {"angle", "dist"}, {0.62f, 2.2f}, "v_perspective", 0, 2, derive_perspective},
    {"line", 346, 1, 2, {"delta", "phi"}, {0.0f, 0.0f}, "v_line", VF_W, 0, nullptr},
    {"holesq", 347, 0, 0, NP, ND, "v_holesq", VF_W, 0, nullptr},
    {"inflateZ_1", 348, 0, 0, NP, ND, "v_inflateZ_1", 0, 0, nullptr},
    {"inflateZ_2", 349, 0, 0, NP, ND, "v_inflateZ_2", 0, 0, nullptr},
    {"inflateZ_3", 350, 0, 0, NP, ND, "v_inflateZ_3", 0, 0, nullptr},
    {"inflateZ_4", 351, 1, 0, NP, ND, "v_inflateZ_4", 0, 0, nullptr},
    {"inflateZ_5", 352, 0, 0, NP, ND, "v_inflateZ_5", 0, 0, nullptr},
    {"inflateZ_6", 353, 0, 0, NP, ND, "v_inflateZ_6", 0, 0, nullptr},
    {"sintrange", 354, 0, 1, {"w"}, {1.0f}, "v_sintrange", VF_REPLACE, 0, nullptr},
    {"foci_3D", 355, 0, 0, NP, ND, "v_foci_3D", 0, 0, nullptr},
    {"asteria", 356, 1, 1, {"alpha"}, {0.0f}, "v_asteria", VF_W, 2, derive_asteria},
    {"estiq", 357, 0, 0, NP, ND, "v_estiq", 0, 0, nullptr},
    {"fdisc", 358, 0, 8, {"ashift", "rshift", "xshift", "yshift", "term1", "term2", "term3", "term4"}, {1.0f, 1.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f}, "v_fdisc", 0, 0, nullptr},
    {"bTransform", 359, 1, 4, {"rotate", "power", "move", "split"}, {0.0f, 1.0f, 0.0f, 0.0f}, "v_bTransform", 0, 0, nullptr},
    {"npolar", 360, 1, 2, {"parity", "n"}, {0.0f, 1.0f}, "v_npolar", VF_W, 4, derive_npolar},
    {"csc_squared", 361, 0, 7, {"csc_div", "cos_div", "tan_div", "csc_pow", "pi_mult", "csc_add", "scaley"}, {1.0f, 1.0f, 1.0f, 0.5f, 0.5f, 0.25f, 1.0f}, "v_csc_squared", 0, 0, nullptr},
    {"hyperbolicellipse", 362, 0, 1, {"a"}, {1.0f}, "v_hyperbolicellipse", VF_REPLACE, 0, nullptr},
    {"layered_spiral", 363, 0, 1, {"radius"}, {1.0f}, "v_layered_spiral", 0, 0, nullptr},
    {"atan2_spirals", 364, 0, 14, {"r_mult", "r_add", "xy2_mult", "xy2_add", "x_mult", "x_add", "yx_div", "yx_add", "yy_div", "yy_add", "sin_add", "y_mult", "r_power", "x2y2_pow"}, {1.5f, 1.0f, 1.125f, 0.132f, 2.0f, 0.25f, 1.0f, 0.0f, 1.25f, 0.0f, 0.0f, 1.0f, 0.5f, 1.0f}, "v_atan2_spirals", 0, 0, nullptr},
    {"gridout2", 365, 0, 4, {"a", "b", "c", "d"}, {1.0f, 1.0f, 1.0f, 1.0f}, "v_gridout2", 0, 0, nullptr},
    {"eJulia", 366, 1, 1, {"power"}, {2.0f}, "v_eJulia", 0, 1, derive_eJulia},
    {"eMotion", 367, 0, 2, {"move", "rotate"}, {0.0f, 0.0f}, "v_eMotion", 0, 0, nullptr},
    {"flower_db", 368, 0, 7, {"petals", "petal_split", "petal_spread", "stem_thickness", "stem_length", "petal_fold_strength", "petal_fold_radius"}, {6.0f, 0.0f, 1.0f, 1.0f, 0.0f, 0.0f, 1.0f}, "v_flower_db", VF_W, 0, nullptr},
    {"julian2", 369, 1, 8, {"power", "dist", "a", "b", "c", "d", "e", "f"}, {0.0f, 1.0f, 1.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f}, "v_julian2", 0, 2, derive_julian2},
    {"mask", 370, 0, 5, {"xshift", "yshift", "ushift", "xscale", "yscale"}, {0.0f, 0.0f, 1.0f, 1.0f, 1.0f}, "v_mask", 0, 0, nullptr},
    {"ovoid3d", 371, 0, 3, {"x", "y", "z"}, {1.0f, 1.0f, 1.0f}, "v_ovoid3d", 0, 0, nullptr},
    {"murl2", 372, 0, 2, {"c", "power"}, {0.1f, 3.0f}, "v_murl2", VF_W, 0, nullptr},
    {"minkQM", 373, 0, 6, {"a", "b", "c", "dd", "e", "f"}, {1.0f, 1.0f, 1.0f, 1.0f, 0.5f, 20.0f}, "v_minkQM", 0, 0, nullptr},
    {"swirl3", 374, 0, 1, {"shift"}, {0.5f}, "v_swirl3", 0, 0, nullptr},
    {"wdisc", 375, 0, 0, NP, ND, "v_wdisc", 0, 0, nullptr},
    {"sph3D", 376, 0, 3, {"x", "y", "z"}, {1.0f, 1.0f, 1.0f}, "v_sph3D", 0, 0, nullptr},
    {"invsquircular", 377, 0, 0, NP, ND, "v_invsquircular", VF_W, 0, nullptr},
    {"sphere_nja", 378, 0, 6, {"circle_a", "circle_b", "shift_x", "shift_y", "shift_z", "stretch"}, {1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 1.0f}, "v_sphere_nja", VF_W, 0, nullptr},
    {"rings", 379, 0, 0, NP, ND, "v_rings", VF_XF | VF_W, 0, nullptr},
    {"rippled", 380, 0, 0, NP, ND, "v_rippled", 0, 0, nullptr},
    {"waffle", 381, 5, 4, {"slices", "xthickness", "ythickness", "rotation"}, {6.0f, 0.5f, 0.5f, 0.0f}, "v_waffle", 0, 2, derive_waffle},
    {"stripfit", 382, 0, 1, {"dx"}, {1.0f}, "v_stripfit", VF_W, 0, nullptr},
    {"q_ode", 383, 0, 12, {"q_ode01", "q_ode02", "q_ode03", "q_ode04", "q_ode05", "q_ode06", "q_ode07", "q_ode08", "q_ode09", "q_ode10", "q_ode11", "q_ode12"}, {0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f}, "v_q_ode", VF_W, 0, nullptr},
    {"ripple", 384, 0, 8, {"frequency", "velocity", "amplitude", "centerx", "centery", "phase", "scale", "fixed_dist_calc"}, {2.0f, 1.0f, 0.5f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f}, "v_ripple", VF_REPLACE, 6, derive_ripple},
    {"scry2", 385, 0, 3, {"sides", "star", "circle"}, {4.0f, 0.0f, 0.0f}, "v_scry2", VF_W, 6, derive_loonie2},
    {"pre_spin_z", 386, 0, 0, NP, ND, "v_pre_spin_z", VF_PRE | VF_W, 0, nullptr},
    {"post_spin_z", 387, 0, 0, NP, ND, "v_post_spin_z", VF_POST | VF_W, 0, nullptr},
    {"post_spherical", 388, 0, 0, NP, ND, "v_post_spherical", VF_POST | VF_W, 0, nullptr},
    {"pre_disc3d", 389, 0, 1, {"pi"}, {3.141592653589793f}, "v_pre_disc3d", VF_PRE | VF_W, 0, nullptr},
    {"waves2_radial", 390, 0, 6, {"w2r_scalex", "w2r_scaley", "w2r_freqx", "w2r_freqy", "w2r_null", "w2r_distance"}, {0.1f, 0.1f, 7.0f, 13.0f, 2.0f, 10.0f}, "v_waves2_radial", 0, 0, nullptr},
    {"spliptic_bs", 391, 1, 2, {"x", "y"}, {0.05f, 0.05f}, "v_spliptic_bs", VF_W, 1, derive_spliptic_bs},
    {"poincare3D", 392, 0, 3, {"r", "a", "b"}, {0.0f, 0.0f, 0.0f}, "v_poincare3D", 0, 10, derive_poincare3D},
    {"pre_sinusoidal3d", 393, 0, 0, NP, ND, "v_pre_sinusoidal3d", VF_PRE | VF_W, 0, nullptr},
    {"pre_blur3D", 394, 8, 0, NP, ND, "v_pre_blur3D", VF_PRE | VF_W, 0, nullptr},
    {"julian3Dx", 395, 1, 8, {"power", "dist", "a", "b", "c", "d", "e", "f"}, {0.0f, 1.0f, 1.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f}, "v_julian3Dx", VF_W, 2, derive_julian3Dx},
    {"rosoni", 396, 0, 7, {"maxiter", "sweetiter", "altshapes", "cutoff", "radius", "dx", "dy"}, {25.0f, 3.0f, 0.0f, 1.0f, 0.4f, 0.6f, 0.0f}, "v_rosoni", 0, 2, derive_rosoni},
    {"seashell3D", 397, 2, 4, {"final_radius", "height", "inner_radius", "nSpirals"}, {0.25f, 3.5f, 0.4f, 3.0f}, "v_seashell3D", 0, 0, nullptr},
    {"hypershift2", 398, 1, 2, {"p", "q"}, {3.0f, 7.0f}, "v_hypershift2", VF_REPLACE, 4, derive_hypershift2},
    {"bwraps7", 399, 0, 5, {"cellsize", "space", "gain", "inner_twist", "outer_twist"}, {1.0f, 0.0f, 2.0f, 0.0f, 0.0f}, "v_bwraps7", 0, 3, derive_bwraps7},
    {"loq", 400, 0, 1, {"base"}, {2.718281828459045f}, "v_loq", 0, 0, nullptr},
    {"pre_bwraps2", 402, 0, 5, {"cellsize", "space", "gain", "inner_twist", "outer_twist"}, {1.0f, 0.0f, 2.0f, 0.0f, 0.0f}, "v_pre_bwraps2", VF_PRE | VF_W, 3, derive_bwraps2},
    {"post_bwraps2", 403, 0, 5, {"cellsize", "space", "gain", "inner_twist", "outer_twist"}, {1.0f, 0.0f, 2.0f, 0.0f, 0.0f}, "v_post_bwraps2", VF_POST | VF_W, 3, derive_bwraps2},
    {"post_heat", 404, 0, 9, {"theta_period", "theta_phase", "theta_amp", "phi_period", "phi_phase", "phi_amp", "r_period", "r_phase", "r_amp"}, {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, "v_post_heat", VF_POST | VF_W, 0, nullptr},
    {"post_rblur", 405, 2, 4, {"strength", "offset", "center_x", "center_y"}, {1.0f, 1.0f, 0.0f, 1.0f}, "v_post_rblur", VF_POST | VF_W, 1, derive_post_rblur},
    {"onion2", 406, 0, 8, {"meeting_pt", "circle_a", "circle_b", "shift_x", "shift_y", "shift_z", "top_crop", "stretch"}, {0.5f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f}, "v_onion2", VF_W, 0, nullptr},
    {"jac_sn", 407, 0, 1, {"jac_sn_k"}, {0.5f}, "v_jac_sn", 0, 0, nullptr},
    {"jac_cn", 408, 0, 1, {"jac_cn_k"}, {0.5f}, "v_jac_cn", 0, 0, nullptr},
    {"jac_dn", 409, 0, 1, {"jac_dn_k"}, {0.5f}, "v_jac_dn", 0, 0, nullptr},
    {"pre_circlecrop", 410, 1, 5, {"radius", "x", "y", "scatter_area", "zero"}, {1.0f, 0.0f, 0.0f, 0.0f, 1.0f}, "v_pre_circlecrop", VF_PRE | VF_W | VF_HIDE, 1, derive_circlecrop},
    {"post_circlecrop", 411, 1, 5, {"radius", "x", "y", "scatter_area", "zero"}, {1.0f, 0.0f, 0.0f, 0.0f, 1.0f}, "v_post_circlecrop", VF_POST | VF_W | VF_HIDE, 1, derive_circlecrop},
    {"circlecrop", 412, 1, 5, {"radius", "x", "y", "scatter_area", "zero"}, {1.0f, 0.0f, 0.0f, 0.0f, 1.0f}, "v_circlecrop", VF_W | VF_HIDE, 1, derive_circlecrop},
    {"exblur", 413, 6, 5, {"dist", "r", "x_origin", "y_origin", "z_origin"}, {0.5f, 0.0f, 0.0f, 0.0f, 0.0f}, "v_exblur", 0, 0, nullptr},
    {"curl_sp", 414, 0, 6, {"pow", "c1", "c2", "sx", "sy", "dc"}, {1.0f, -0.01f, 0.03f, 0.0f, 0.0f, 0.0f}, "v_curl_sp", VF_W, 4, derive_curl_sp},
    {"extrude", 415, 1, 1, {"root_face"}, {0.5f}, "v_extrude", 0, 0, nullptr},
    {"minkowskope", 417, 0, 6, {"separation", "frequencyx", "frequencyy", "amplitude", "perturbation", "damping"}, {0.5f, 1.5f, 1.0f, 0.5f, 0.3f, 0.0f}, "v_minkowskope", 0, 2, derive_minkowskope},
    {"glynnlissa", 418, 4, 11, {"radius", "radius1", "thickness", "phi1", "a", "b", "width", "phase", "scale", "pow", "contrast"}, {1.0f, 0.5f, 1.0f, 0.0f, 3.0f, 2.0f, 0.0f, 0.0f, 0.71f, 1.5f, 0.5f}, "v_glynnlissa", 0, 3, derive_glynnlissa},
    {"lazysensen", 421, 0, 3, {"scale_x", "scale_y", "scale_z"}, {1.0f, 1.0f, 0.0f}, "v_lazysensen", 0, 0, nullptr},
    {"spherecrop", 422, 1, 6, {"radius", "x", "y", "z", "scatter_area", "zero"}, {1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f}, "v_spherecrop", VF_W | VF_HIDE, 1, derive_spherecrop},
    {"xheart_blur_wf", 423, 2, 2, {"angle", "ratio"}, {0.0f, 0.0f}, "v_xheart_blur_wf", 0, 3, derive_xheart_blur_wf},
    {"circleLinear", 425, 0, 8, {"Sc", "K", "Dens1", "Dens2", "Reverse", "X", "Y", "Seed"}, {1.0f, 0.5f, 0.5f, 0.5f, 1.0f, 10.0f, 10.0f, 0.0f}, "v_circleLinear", 0, 0, nullptr},
    {"cannabiscurve_wf", 426, 1, 1, {"filled"}, {1.0f}, "v_cannabiscurve_wf", 0, 0, nullptr},
    {"spherical3D_wf", 427, 0, 2, {"invert", "exponent"}, {0.0f, 2.0f}, "v_spherical3D_wf", 0, 1, derive_spherical3D_wf},
    {"heart_wf", 429, 0, 5, {"scale_x", "scale_t", "shift_t", "scale_r_left", "scale_r_right"}, {1.0f, 1.0f, 0.0f, 1.0f, 1.0f}, "v_heart_wf", 0, 0, nullptr},
    {"post_ztranslate_wf", 430, 0, 0, NP, ND, "v_post_ztranslate_wf", VF_POST, 0, nullptr},
    {"cpow3_wf", 434, 3, 7, {"r", "a", "divisor", "spread", "discrete_spread", "spread2", "offset2"}, {1.0f, 0.1f, 1.0f, 1.0f, 1.0f, 0.0f, 1.0f}, "v_cpow3_wf", 0, 7, derive_cpow3_wf},
    {"clifford_js", 435, 0, 4, {"a", "b", "c", "d"}, {-1.4f, 1.6f, 1.0f, 0.7f}, "v_clifford_js", 0, 0, nullptr},
    {"svensson_js", 436, 0, 4, {"a", "b", "c", "d"}, {1.4f, 1.56f, 1.4f, -6.56f}, "v_svensson_js", VF_REPLACE, 0, nullptr},
    {"sattractor_js", 437, 2, 1, {"m"}, {10.0f}, "v_sattractor_js", 0, 0, nullptr},
    {"threepoint_js", 438, 2, 0, NP, ND, "v_threepoint_js", 0, 0, nullptr},
    {"woggle_js", 440, 1, 1, {"m"}, {2.0f}, "v_woggle_js", 0, 0, nullptr},
    {"lace_js", 441, 1, 0, NP, ND, "v_lace_js", 0, 0, nullptr},
    {"wallpaper_js", 442, 1, 3, {"a", "b", "c"}, {1.156f, -0.28f, 21.288f}, "v_wallpaper_js", VF_W, 0, nullptr},
    {"hadamard_js", 443, 2, 0, NP, ND, "v_hadamard_js", 0, 0, nullptr},
    {"invtree_js", 444, 2, 0, NP, ND, "v_invtree_js", 0, 0, nullptr},
    {"epispiral_wf", 446, 0, 1, {"waves"}, {4.0f}, "v_epispiral_wf", 0, 0, nullptr},
    {"cloverleaf_wf", 447, 1, 1, {"filled"}, {1.0f}, "v_cloverleaf_wf", 0, 0, nullptr},
    {"rose_wf", 448, 1, 3, {"amp", "waves", "filled"}, {0.5f, 4.0f, 0.0f}, "v_rose_wf", 0, 0, nullptr},
    {"bubble_wf", 449, 0, 0, NP, ND, "v_bubble_wf", 0, 0, nullptr},
    {"waves2_wf", 452, 0, 8, {"scalex", "scaley", "freqx", "freqy", "use_cos_x", "use_cos_y", "dampx", "dampy"}, {0.25f, 0.5f, 1.5707963267948966f, 0.7853981633974483f, 1.0f, 0.0f, 0.0f, 0.0f}, "v_waves2_wf", 0, 2, derive_waves_wf},
    {"waves3_wf", 453, 0, 8, {"scalex", "scaley", "freqx", "freqy", "use_cos_x", "use_cos_y", "dampx", "dampy"}, {0.25f, 0.5f, 1.5707963267948966f, 0.7853981633974483f, 1.0f, 0.0f, 0.0f, 0.0f}, "v_waves3_wf", 0, 2, derive_waves_wf},
    {"waves4_wf", 454, 0, 8, {"scalex", "scaley", "freqx", "freqy", "use_cos_x", "use_cos_y", "dampx", "dampy"}, {0.25f, 0.5f, 1.5707963267948966f, 0.7853981633974483f, 1.0f, 0.0f, 0.0f, 0.0f}, "v_waves4_wf", 0, 2, derive_waves_wf},
    {"dinis_surface_wf", 455, 0, 2, {"a", "b"}, {0.8f, 0.2f}, "v_dinis_surface_wf", 0, 0, nullptr},
    {"pointgrid_wf", 456, 2, 8, {"xmin", "xmax", "xcount", "ymin", "ymax", "ycount", "distortion", "seed"}, {-3.0f, 3.0f, 32.0f, -3.0f, 3.0f, 32.0f, 2.3f, 1234.0f}, "v_pointgrid_wf", 0, 2, derive_pointgrid_wf},
    {"apocarpet_js", 458, 1, 0, NP, ND, "v_apocarpet_js", 0, 0, nullptr},
    {"pre_rect_wf", 463, 2, 4, {"x0", "x1", "y0", "y1"}, {-0.5f, 0.5f, -0.5f, 0.5f}, "v_pre_rect_wf", VF_PRE | VF_W, 2, derive_pre_rect_wf},
    {"affine3D", 464, 0, 15, {"translateX", "translateY", "translateZ", "scaleX", "scaleY", "scaleZ", "rotateX", "rotateY", "rotateZ", "shearXY", "shearXZ", "shearYX", "shearYZ", "shearZX", "shearZY"}, {0.0f, 0.0f, 0.0f, 1.0f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, "v_affine3D", 0, 7, derive_affine3D},
    {"truchet2", 465, 0, 7, {"exponent1", "exponent2", "width1", "width2", "scale", "seed", "inverse"}, {1.0f, 2.0f, 0.5f, 0.5f, 10.0f, 50.0f, 0.0f}, "v_truchet2", 0, 0, nullptr},
    {"pre_wave3D_wf", 468, 0, 7, {"axis", "wavelen", "phase", "damping", "centre_x", "centre_y", "centre_z"}, {0.0f, 0.5f, 0.0f, 0.01f, 0.0f, 0.0f, 0.0f}, "v_pre_wave3D_wf", VF_PRE | VF_W, 0, nullptr},
    {"siercarpet_js", 473, 1, 1, {"m"}, {3.0f}, "v_siercarpet_js", 0, 0, nullptr},
    {"popcorn2_3D", 474, 0, 4, {"popcorn2_3D_x", "popcorn2_3D_y", "popcorn2_3D_z", "popcorn2_3D_c"}, {0.1f, 0.1f, 0.1f, 3.0f}, "v_popcorn2_3D", 0, 0, nullptr},
    {"plusrecip", 476, 0, 2, {"ar", "ai"}, {4.0f, 0.0f}, "v_plusrecip", 0, 0, nullptr},
    {"gamma", 477, 0, 0, NP, ND, "v_gamma", 0, 0, nullptr},
    {"bubbleT3D", 478, 0, 6, {"number_of_stripes", "ratio_of_stripes", "angle_of_hole", "exponent_z", "symmetry_z", "modus_blur"}, {0.0f, 1.0f, 0.0f, 1.0f, 0.0f, 0.0f}, "v_bubbleT3D", 0, 7, derive_bubbleT3D},
    {"waves2b", 479, 0, 10, {"freqx", "freqy", "pwx", "pwy", "scalex", "scaleinfx", "scaley", "scaleinfy", "unity", "jacok"}, {2.0f, 2.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 0.25f}, "v_waves2b", 0, 2, derive_waves2b},
    {"z", 489, 0, 13, {"hypergon", "hypergon_n", "hypergon_r", "star", "star_n", "star_slope", "lituus", "lituus_a", "super_shape", "super_m", "super_n1", "super_n2", "super_n3"}, {0.0f, 4.0f, 1.0f, 0.0f, 5.0f, 2.0f, 0.0f, 1.0f, 0.0f, 1.0f, 1.0f, 1.0f, 0.0f}, "v_z", 0, 7, derive_z},
    {"w", 490, 0, 14, {"angle", "hypergon", "hypergon_n", "hypergon_r", "star", "star_n", "star_slope", "lituus", "lituus_a", "super_shape", "super_m", "super_n1", "super_n2", "super_n3"}, {0.0f, 0.0f, 4.0f, 1.0f, 0.0f, 5.0f, 2.0f, 0.0f, 1.0f, 0.0f, 1.0f, 1.0f, 1.0f, 0.0f}, "v_w", 0, 7, derive_w},
    {"harmonograph_js", 496, 1, 18, {"seed", "time", "a1", "f1", "p1", "d1", "a2", "f2", "p2", "d2", "a3", "f3", "p3", "d3", "a4", "f4", "p4", "d4"}, {1234.0f, 100.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, "v_harmonograph_js", 0, 0, nullptr},
    {"klein_group", 501, 1, 6, {"a_re", "a_im", "b_re", "b_im", "recipe", "avoid_reversal"}, {2.0f, 0.0f, 2.0f, 0.0f, 0.0f, 1.0f},
     "v_klein_group", VF_W, 16, derive_klein_group, 1, 1},
    {"subflame_wf", 502, 0, 8, {"subflame_id", "scale", "angle", "offset_x", "offset_y", "offset_z", "colorscale_z", "color_mode"},
     {0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, -1.0f}, "v_subflame_wf", VF_W | VF_DC | VF_SUB, 2, derive_subflame, 6, 0},
    {"pre_subflame_wf", 503, 0, 8, {"subflame_id", "scale", "angle", "offset_x", "offset_y", "offset_z", "colorscale_z", "color_mode"},
     {0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, -1.0f}, "v_pre_subflame_wf", VF_PRE | VF_DC | VF_SUB, 2, derive_subflame, 6, 0},
    {"linear3D", 533, 0, 0, NP, ND, "v_linear3D", 0, 0, nullptr},

    {"sym_ng1", 544, 1, 2, {"stepx", "stepy"}, {0.5f, 0.5f}, "v_sym_ng1", 0, 0, nullptr},
    {"sym_ng2", 545, 1, 2, {"stepx", "stepy"}, {2.0f, 2.0f}, "v_sym_ng2", 0, 0, nullptr},
    {"sym_ng3", 546, 1, 3, {"sepx", "sepy", "step"}, {0.5f, 0.0f, 2.0f}, "v_sym_ng3", 0, 0, nullptr},
    {"sym_ng4", 547, 1, 4, {"sepx", "sepy", "stepx", "stepy"}, {0.0f, 0.0f, 0.0f, 0.0f}, "v_sym_ng4", 0, 0, nullptr},
    {"sym_ng5", 548, 1, 3, {"sepx", "sepy", "stepx"}, {0.0f, 0.0f, 0.0f}, "v_sym_ng5", 0, 0, nullptr},
    {"sym_ng6", 549, 1, 3, {"sepy", "stepx", "stepy"}, {0.1f, 1.0f, 1.0f}, "v_sym_ng6", 0, 0, nullptr},
    {"sym_ng7", 550, 1, 2, {"sepx", "sepy"}, {0.0f, 0.0f}, "v_sym_ng7", 0, 0, nullptr},
    {"sym_ng8", 551, 1, 4, {"sepx", "sepy", "skewx", "skewy"}, {0.0f, 0.0f, 0.0f, 0.0f}, "v_sym_ng8", 0, 0, nullptr},
    {"sym_ng9", 552, 1, 2, {"sepx", "sepy"}, {0.0f, 0.0f}, "v_sym_ng9", 0, 0, nullptr},
    {"sym_ng10", 553, 1, 3, {"space", "spacex", "spacey"}, {0.0f, 0.0f, 0.0f}, "v_sym_ng10", 0, 0, nullptr},
    {"sym_ng11", 554, 1, 5, {"space", "spacex", "spacey", "stepx", "stepy"}, {0.0f, 0.0f, 0.0f, 1.5f, 1.5f}, "v_sym_ng11", 0, 0, nullptr},
    {"sym_ng12", 555, 1, 3, {"space", "spacex", "spacey"}, {0.0f, 0.0f, 0.0f}, "v_sym_ng12", 0, 0, nullptr},
    {"sym_ng13", 556, 1, 3, {"radius", "stepx", "stepy"}, {0.0f, 0.0f, 0.0f}, "v_sym_ng13", 0, 0, nullptr},
    {"sym_ng14", 557, 1, 3, {"radius", "stepx", "stepy"}, {0.0f, 0.0f, 0.0f}, "v_sym_ng14", 0, 0, nullptr},
    {"sym_ng15", 558, 1, 3, {"radius", "stepx", "stepy"}, {0.0f, 0.0f, 0.0f}, "v_sym_ng15", 0, 0, nullptr},
    {"sym_ng16", 559, 1, 3, {"radius", "stepx", "stepy"}, {0.0f, 0.0f, 0.0f}, "v_sym_ng16", 0, 0, nullptr},
    {"sym_ng17", 560, 1, 3, {"radius", "stepx", "stepy"}, {0.0f, 0.0f, 0.0f}, "v_sym_ng17", 0, 0, nullptr},
    {"sym_bg1", 561, 1, 2, {"stepx", "stepy"}, {0.0f, 0.0f}, "v_sym_bg1", 0, 0, nullptr},
    {"sym_bg2", 562, 1, 2, {"stepx", "stepy"}, {0.0f, 0.0f}, "v_sym_bg2", 0, 0, nullptr},
    {"sym_bg3", 563, 1, 2, {"stepx", "stepy"}, {0.0f, 0.0f}, "v_sym_bg3", 0, 0, nullptr},
    {"sym_bg4", 564, 1, 2, {"stepx", "stepy"}, {0.0f, 0.0f}, "v_sym_bg4", 0, 0, nullptr},
    {"sym_bg5", 565, 1, 2, {"stepx", "stepy"}, {0.0f, 0.0f}, "v_sym_bg5", 0, 0, nullptr},
    {"sym_bg6", 566, 1, 2, {"stepx", "stepy"}, {0.0f, 0.0f}, "v_sym_bg6", 0, 0, nullptr},
    {"sym_bg7", 567, 1, 2, {"stepx", "stepy"}, {0.0f, 0.0f}, "v_sym_bg7", 0, 0, nullptr},
    {"pRose3D", 568, 2, 16, {"l", "k", "c", "z1", "z2", "refSc", "opt", "optSc", "opt3", "transp", "dist", "wagsc", "srvsc", "f", "wigsc", "offset"}, {1.0f, 6.0f, 0.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 0.0f, 0.5f, 1.0f, 0.0f, 0.0f, 3.0f, 0.0f, 0.0f}, "v_pRose3D", 0, 0, nullptr},
    {"cut_hextruchetflow", 569, 2, 5, {"randomize", "mode", "grid", "zoom", "invert"}, {0.0f, 1.0f, 0.0f, 10.0f, 0.0f}, "v_cut_hextruchetflow", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_sqcir", 570, 2, 4, {"mode", "zoom", "invert", "power"}, {1.0f, 2.0f, 0.0f, 2.0f}, "v_cut_sqcir", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_yuebing", 571, 2, 5, {"mode", "zoom", "invert", "p1", "p2"}, {1.0f, 0.25f, 0.0f, 2.0f, 25.0f}, "v_cut_yuebing", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_vasarely", 572, 2, 4, {"mode", "zoom", "invert", "size"}, {1.0f, 1.0f, 0.0f, 0.5f}, "v_cut_vasarely", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_sincos", 573, 2, 5, {"seed", "mode", "time", "zoom", "invert"}, {1000.0f, 1.0f, 0.9f, 0.5f, 0.0f}, "v_cut_sincos", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_chains", 574, 2, 5, {"shiftX", "shiftY", "mode", "zoom", "invert"}, {0.0f, 0.0f, 1.0f, 2.5f, 0.0f}, "v_cut_chains", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_hexdots", 575, 2, 4, {"mode", "size", "zoom", "invert"}, {1.0f, 0.5f, 4.0f, 0.0f}, "v_cut_hexdots", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_booleans", 576, 2, 5, {"seed", "mode", "type", "zoom", "invert"}, {1000.0f, 1.0f, 0.0f, 250.0f, 0.0f}, "v_cut_booleans", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_sqsplits", 577, 2, 5, {"seed", "mode", "time", "zoom", "invert"}, {1000.0f, 1.0f, 0.9f, 2.0f, 0.0f}, "v_cut_sqsplits", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_btree", 578, 2, 6, {"seed", "time", "thickness", "zoom", "mode", "invert"}, {0.0f, 1.0f, 5.0f, 1.0f, 1.0f, 1.0f}, "v_cut_btree", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_fractal", 579, 2, 6, {"seed", "mode", "time", "iters", "zoom", "invert"}, {0.0f, 1.0f, 0.0f, 30.0f, 1.0f, 0.0f}, "v_cut_fractal", VF_REPLACE | VF_HIDE, 2, derive_cut_fractal},
    {"cut_glypho", 580, 2, 6, {"mode", "zoom", "invert", "f1", "f2", "f3"}, {1.0f, 1.0f, 0.0f, 0.115f, 0.75f, 1.5f}, "v_cut_glypho", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_circdes", 581, 2, 5, {"seed", "mode", "time", "zoom", "invert"}, {1000.0f, 1.0f, 0.0f, 10.0f, 0.0f}, "v_cut_circdes", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_snowflake", 582, 2, 6, {"seed", "mode", "time", "level", "zoom", "invert"}, {1000.0f, 1.0f, 0.0f, 10.0f, 10.0f, 0.0f}, "v_cut_snowflake", VF_REPLACE | VF_HIDE, 1, derive_cut_snowflake},
    {"cut_jigsaw", 583, 2, 5, {"seed", "time", "mode", "zoom", "invert"}, {1000.0f, 0.0f, 1.0f, 4.0f, 0.0f}, "v_cut_jigsaw", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_rgrid", 584, 2, 4, {"mode", "zoom", "invert", "angle"}, {1.0f, 7.0f, 0.0f, 0.0f}, "v_cut_rgrid", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_x", 585, 2, 4, {"mode", "zoom", "invert", "size"}, {1.0f, 1.0f, 0.0f, 0.1f}, "v_cut_x", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_metaballs", 586, 2, 4, {"mode", "zoom", "invert", "time"}, {1.0f, 7.0f, 0.0f, 0.0f}, "v_cut_metaballs", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_kaleido", 587, 2, 6, {"seed", "mode", "time", "n", "zoom", "invert"}, {1000.0f, 1.0f, 0.0f, 6.0f, 0.5f, 0.0f}, "v_cut_kaleido", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_spiral", 588, 2, 4, {"time", "mode", "zoom", "invert"}, {0.0f, 1.0f, 2.5f, 0.0f}, "v_cut_spiral", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_swarp", 589, 2, 6, {"seed", "mode", "time", "type", "zoom", "invert"}, {1000.0f, 1.0f, 0.0f, 0.0f, 1.0f, 0.0f}, "v_cut_swarp", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_apollonian", 590, 2, 4, {"mode", "levels", "zoom", "invert"}, {1.0f, 4.0f, 2.0f, 0.0f}, "v_cut_apollonian", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_zigzag", 591, 2, 5, {"mode", "xpar", "ypar", "zoom", "invert"}, {1.0f, 1.0f, 2.0f, 2.0f, 0.0f}, "v_cut_zigzag", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_bricks", 592, 2, 5, {"seed", "mode", "size", "zoom", "invert"}, {1000.0f, 1.0f, 0.9f, 3.0f, 0.0f}, "v_cut_bricks", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_web", 593, 2, 5, {"seed", "time", "mode", "thick", "invert"}, {1000.0f, 0.0f, 1.0f, 0.05f, 1.0f}, "v_cut_web", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_tileillusion", 595, 2, 4, {"time", "mode", "zoom", "invert"}, {0.0f, 1.0f, 15.0f, 0.0f}, "v_cut_tileillusion", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_pattern", 596, 2, 5, {"seed", "mode", "time", "zoom", "invert"}, {1000.0f, 1.0f, 0.9f, 0.5f, 0.0f}, "v_cut_pattern", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"cut_celtic", 597, 2, 3, {"mode", "zoom", "invert"}, {1.0f, 5.0f, 0.0f}, "v_cut_celtic", VF_REPLACE | VF_HIDE, 0, nullptr},
    {"solid_sphere", 605, 2, 5, {"radius", "thickness", "cx", "cy", "cz"}, {1.0f, 0.1f, 0.0f, 0.0f, 0.0f}, "v_solid_sphere", 0, 0, nullptr},
    {"matrix3D", 643, 0, 12, {"xx", "xy", "xz", "yx", "yy", "yz", "zx", "zy", "zz", "tx", "ty", "tz"}, {1.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f}, "v_matrix3D", 0, 0, nullptr},};
#undef NP
#undef ND

const VarDef* registry_find(const std::string& name) {
    for (const auto& v : kRegistry) if (name == v.name) return &v;
    return nullptr;
}

const std::vector<const VarDef*>& registry_all() {
    static std::vector<const VarDef*> all = [] {
        std::vector<const VarDef*> a;
        for (const auto& v : kRegistry) a.push_back(&v);
        return a;
    }();
    return all;
}

float XForm::param(const VarDef* v, int j) const {
    std::string key = std::string(v->name) + "." + v->pname[j];
    for (auto& p : params) if (p.first == key) return p.second;
    return v->pdef[j];
}

void XForm::slot_values(const VarDef* v, float* out) const {
    for (int j = 0; j < v->nparams; ++j) out[j] = param(v, j);
    if (v->nderived > 0) v->derive(out, out + v->nparams);
}

float XForm::var_weight(const VarDef* v) const {
    for (auto& p : vars) if (p.first == v) return p.second;
    return 0.0f;
}

namespace {

[[noreturn]] void fail(const std::string& s) { throw std::runtime_error(s); }

float num_field(const Json& o, const char* k, bool required, float dflt) {
    const Json* v = o.get(k);
    if (!v || v->kind == Json::Null) {
        if (required) fail(std::string("missing field `") + k + "`");
        return dflt;
    }
    if (v->kind != Json::Number) fail(std::string("`") + k + "` is not a number");
    return (float)v->num;
}

XForm parse_transform(const Json& t) {
    if (t.kind != Json::Object) fail("a transform is not an object");
    XForm x;
    x.a = num_field(t, "a", true, 0); x.b = num_field(t, "b", true, 0); x.c = num_field(t, "c", true, 0);
    x.d = num_field(t, "d", true, 0); x.e = num_field(t, "e", true, 0); x.f = num_field(t, "f", true, 0);
    x.weight = num_field(t, "weight", true, 0);
    // color: a palette position, or the old [r,g,b] form averaged (transforms.rs:1440-1458).
    const Json* c = t.get("color");
    if (!c) fail("missing field `color`");
    if (c->kind == Json::Number) x.color = (float)c->num;
    else if (c->kind == Json::Array && c->arr.size() >= 3) {
        float r = (float)c->arr[0]->num, g = (float)c->arr[1]->num, b = (float)c->arr[2]->num;
        x.color = (r + g + b) / 3.0f;
    } else x.color = 0.5f;
    x.speed = num_field(t, "color_speed", false, 0.0f);       // transforms.rs:1538
    x.opacity = num_field(t, "opacity", false, 1.0f);
    x.direct_color = num_field(t, "direct_color", false, 0.0f);      // transforms.rs:1533-1540
    x.post = t.bool_or("post_affine_enabled", false);        // transforms.rs:1542
    x.pa = num_field(t, "post_a", false, 1); x.pb = num_field(t, "post_b", false, 0);
    x.pc = num_field(t, "post_c", false, 0); x.pd = num_field(t, "post_d", false, 1);
    x.pe = num_field(t, "post_e", false, 0); x.pf = num_field(t, "post_f", false, 0);
    const Json* vs = t.get("variations");
    if (!vs || vs->kind != Json::Object) fail("missing field `variations`");
    std::vector<std::pair<const VarDef*, float>> found;
    for (auto& kv : vs->obj) {
        const VarDef* d = registry_find(kv.first);
        if (!d) fail("variation `" + kv.first + "` is not supported by this build");
        if (kv.second->kind != Json::Number) fail("variation weight of `" + kv.first + "` is not a number");
        found.emplace_back(d, (float)kv.second->num);
    }
    // Dispatch order (transforms.rs:668-682): `variation_order` first, then
    // the registry's order.
    std::vector<const VarDef*> order;
    if (const Json* vo = t.get("variation_order"); vo && vo->kind == Json::Array) {
        for (auto& e : vo->arr) {
            if (e->kind != Json::String) continue;
            const VarDef* d = registry_find(e->str);
            if (!d) continue;
            bool present = false;
            for (auto& p : found) present |= p.first == d;
            if (present && std::find(order.begin(), order.end(), d) == order.end()) order.push_back(d);
        }
    }
    for (const VarDef* d : registry_all())
        for (auto& p : found)
            if (p.first == d && std::find(order.begin(), order.end(), d) == order.end()) order.push_back(d);
    for (const VarDef* d : order)
        for (auto& p : found) if (p.first == d) x.vars.emplace_back(d, p.second);
    if (const Json* vp = t.get("variation_params"); vp && vp->kind == Json::Object)
        for (auto& kv : vp->obj) if (kv.second->kind == Json::Number) x.params.emplace_back(kv.first, (float)kv.second->num);
    if (const Json* fa = t.get("final_attachments"); fa && fa->kind == Json::Array)
        for (auto& e : fa->arr) if (e->kind == Json::Number) x.final_att.push_back((int)e->num);
    if (const Json* la = t.get("linked_attachments"); la && la->kind == Json::Array)
        for (auto& e : la->arr) if (e->kind == Json::Number) x.linked_att.push_back((int)e->num);
    return x;
}

int mode_code(const std::string& s, const char* const* names, int n, const char* what) {
    for (int i = 0; i < n; ++i) {
        const char* a = names[2 * i];
        const char* b = names[2 * i + 1];
        if (s == a || s == b) return i;
    }
    fail(std::string("unknown ") + what + " `" + s + "`");
}

}  // namespace

// Whether the xaos walk, not the first pick, decides which closed group of
// the chain an orbit ends in (xaos.rs:66-123, restated): transitions go
// where weight x xaos > 0 (a row with none goes to transform 0); a closed
// group is a set the chain never leaves; a start is any transform of
// positive weight.
static bool xaos_walk_splits_orbits(const Flame& F) {
    const size_t n = F.xf.size();
    if (F.xaos.empty() || n == 0) return false;
    std::vector<std::vector<size_t>> next(n);
    for (size_t i = 0; i < n; ++i) {
        for (size_t j = 0; j < n; ++j)
            if (std::max(F.xf[j].weight, 0.0f) * F.xaos[i * n + j] > 0.0f) next[i].push_back(j);
        if (next[i].empty()) next[i].push_back(0);
    }
    std::vector<std::vector<char>> reach(n, std::vector<char>(n, 0));
    for (size_t s = 0; s < n; ++s) {
        std::vector<size_t> stack{s};
        reach[s][s] = 1;
        while (!stack.empty()) {
            const size_t i = stack.back();
            stack.pop_back();
            for (size_t j : next[i]) if (!reach[s][j]) { reach[s][j] = 1; stack.push_back(j); }
        }
    }
    std::vector<char> first(n), live(n, 0);
    for (size_t i = 0; i < n; ++i) first[i] = F.xf[i].weight > 0.0f;
    for (size_t i = 0; i < n; ++i)
        if (first[i]) for (size_t j = 0; j < n; ++j) live[j] |= reach[i][j];
    std::vector<size_t> closed;
    for (size_t i = 0; i < n; ++i) {
        if (!live[i]) continue;
        bool cl = true, lowest = true;
        for (size_t j = 0; j < n; ++j) cl &= !reach[i][j] || reach[j][i];
        for (size_t j = 0; j < i; ++j) lowest &= !(reach[i][j] && reach[j][i]);
        if (cl && lowest) closed.push_back(i);
    }
    if (closed.size() < 2) return false;
    for (size_t i = 0; i < n; ++i) {
        if (!first[i]) continue;
        int k = 0;
        for (size_t c : closed) k += reach[i][c] ? 1 : 0;
        if (k > 1) return true;
    }
    return false;
}

Flame parse_config(const Json& cfg) {
    if (cfg.kind != Json::Object) fail("the config is not a JSON object");
    const Json* fl = cfg.get("flame");
    if (!fl || fl->kind != Json::Object) fail("missing field `flame`");
    Flame F;
    std::string rm = cfg.string_or("render_mode", fl->string_or("render_mode", "TwoD"));
    if (rm != "TwoD" && rm != "2d" && rm != "two_d") fail("render mode `" + rm + "` is not supported by this build (2-D flames only)");
    const Json* ts = fl->get("transforms");
    if (!ts || ts->kind != Json::Array) fail("missing field `transforms`");
    for (auto& t : ts->arr) F.xf.push_back(parse_transform(*t));
    if (const Json* lt = fl->get("linked_transforms"); lt && lt->kind == Json::Array)
        for (auto& t : lt->arr) F.lnk.push_back(parse_transform(*t));
    // Xaos (utilities.wgsl:106-137): read when some weight differs from 1
    // (xaos.rs:29-40); entries beyond the matrix are 1 (get_xaos, xaos.rs:128-135).
    if (const Json* xa = fl->get("xaos"); xa && xa->kind == Json::Array) {
        const size_t n = F.xf.size();
        std::vector<float> m(n * n, 1.0f);
        bool any = false;
        for (size_t i = 0; i < xa->arr.size(); ++i) {
            const Json* row = xa->arr[i].get();
            if (row->kind != Json::Array) fail("xaos rows must be arrays");
            for (size_t j = 0; j < row->arr.size(); ++j) {
                if (row->arr[j]->kind != Json::Number) fail("xaos weights must be numbers");
                const float v = (float)row->arr[j]->num;
                any |= std::fabs(v - 1.0f) > 1e-6f;
                if (i < n && j < n) m[i * n + j] = v;
            }
        }
        if (any) {
            if (n > 64) fail("xaos over more than 64 transforms is not supported by this build");
            F.xaos = m;
            if (xaos_walk_splits_orbits(F)) F.orbit_refresh = 4;           // ORBIT_REFRESH_PERIOD
        }
    }
    if (const Json* so = fl->get("solo_transform"); so && so->kind == Json::Number) {
        if (!(so->num >= 0.0) || so->num != std::floor(so->num)) fail("`solo_transform` is not a usize");
        F.solo = so->num < 1e9 ? (int)so->num : 1000000000;
    }
    if (const Json* ft = fl->get("final_transforms"); ft && ft->kind == Json::Array)
        for (auto& t : ft->arr) F.fin.push_back(parse_transform(*t));
    // A legacy singular final joins the pool attached to every normal
    // (transforms.rs:2253-2266).
    if (const Json* lf = fl->get("final_transform"); lf && lf->kind == Json::Object) {
        int idx = (int)F.fin.size();
        F.fin.push_back(parse_transform(*lf));
        for (auto& x : F.xf)
            if (std::find(x.final_att.begin(), x.final_att.end(), idx) == x.final_att.end()) x.final_att.push_back(idx);
    }
    if (F.xf.empty()) fail("the flame has no transforms");
    if (F.xf.size() > 128)
        fail("TooLarge: the flame has " + std::to_string(F.xf.size()) + " transforms; the renderer holds 128");
    // Attachment lists (GpuAttachmentList::from_transform, gpu/buffers.rs:621-660):
    // indices past their pool dropped, at most kMaxAttach kept.
    auto clean = [](std::vector<int>& att, size_t pool) {
        std::vector<int> out;
        for (int a : att) {
            if ((int)out.size() >= kMaxAttach) break;
            if (a >= 0 && (size_t)a < pool) out.push_back(a);
        }
        att = out;
    };
    for (auto& x : F.xf) { clean(x.final_att, F.fin.size()); clean(x.linked_att, F.lnk.size()); }
    // Attachments only a normal transform carries.
    for (auto& x : F.lnk) { x.final_att.clear(); x.linked_att.clear(); }
    for (auto& x : F.fin) { x.final_att.clear(); x.linked_att.clear(); }
    F.fin_chain = F.xf[0].final_att;
    for (auto& x : F.xf) F.fin_uniform = F.fin_uniform && x.final_att == F.fin_chain;
    if (!F.fin_uniform) F.fin_chain.clear();
    std::vector<char> fu(F.fin.size(), 0), lu(F.lnk.size(), 0);
    for (auto& x : F.xf) {
        for (int a : x.final_att) fu[(size_t)a] = 1;
        for (int a : x.linked_att) lu[(size_t)a] = 1;
    }
    for (size_t i = 0; i < fu.size(); ++i) if (fu[i]) F.fin_used.push_back((int)i);
    for (size_t i = 0; i < lu.size(); ++i) if (lu[i]) F.lnk_used.push_back((int)i);
    if (F.fin_used.size() > 16) fail("more than 16 attached final transforms are not supported by this build");
    if (F.lnk_used.size() > 16) fail("more than 16 attached linked transforms are not supported by this build");
    // Post-symmetry (transforms.rs:2149-2167; serde: `ty` lowercase, the
    // other fields required when the object is present).
    if (const Json* ps = fl->get("post_symmetry"); ps && ps->kind == Json::Object) {
        const std::string ty = ps->string_or("ty", "none");
        F.sym.kind = ty == "none" ? 0 : ty == "xaxis" ? 1 : ty == "yaxis" ? 2 : ty == "point" ? 3 : -1;
        if (F.sym.kind < 0) fail("unknown variant `" + ty + "`, expected one of `none`, `xaxis`, `yaxis`, `point`");
        const float order = num_field(*ps, "order", true, 3.0f);
        if (!(order >= 0.0f) || order != std::floor(order)) fail("`order` is not a u32");
        F.sym.order = (int)std::min(std::max(order, 1.0f), 32.0f);           // clamp(1, 32): buffers.rs:958
        F.sym.cx = num_field(*ps, "center_x", true, 0.0f);
        F.sym.cy = num_field(*ps, "center_y", true, 0.0f);
        F.sym.distance = num_field(*ps, "distance", true, 1.25f);
        const float deg = num_field(*ps, "rotation_deg", true, 6.0f);
        const float rads_per_deg = 3.14159265358979323846f / 180.0f;      // f32::to_radians
        F.sym.rotation = deg * rads_per_deg;
    }
    // Subflames (fractal_config.rs:178-190; gpu/buffers.rs:36-56, 230-253):
    // each an inner flame's normals and finals (a legacy singular final
    // joins its finals); their own xaos and subflames are not read.
    if (const Json* sfs = fl->get("subflames"); sfs && sfs->kind == Json::Array) {
        if (sfs->arr.size() > 8) fail("more than 8 subflames (MAX_SUBFLAMES)");
        size_t total = 0;
        for (auto& sj : sfs->arr) {
            if (sj->kind != Json::Object) fail("a subflame is not an object");
            SubFlame S;
            if (const Json* st = sj->get("transforms"); st && st->kind == Json::Array)
                for (auto& t : st->arr) S.xf.push_back(parse_transform(*t));
            if (const Json* ft = sj->get("final_transforms"); ft && ft->kind == Json::Array)
                for (auto& t : ft->arr) S.fin.push_back(parse_transform(*t));
            if (const Json* lf = sj->get("final_transform"); lf && lf->kind == Json::Object) S.fin.push_back(parse_transform(*lf));
            total += S.xf.size() + S.fin.size();
            F.sub.push_back(std::move(S));
        }
        if (total > 256) fail("TooLarge: the subflames have " + std::to_string(total) + " transforms; the renderer holds 256");
    }
    // Local variation order (transforms.rs:2297-2319): normals, linked,
    // finals, then each subflame's.
    auto absorb = [&](const XForm& x) {
        for (auto& p : x.vars)
            if (std::find(F.local.begin(), F.local.end(), p.first) == F.local.end()) F.local.push_back(p.first);
    };
    for (auto& x : F.xf) absorb(x);
    for (auto& x : F.lnk) absorb(x);
    for (auto& x : F.fin) absorb(x);
    for (auto& S : F.sub) {
        for (auto& x : S.xf) absorb(x);
        for (auto& x : S.fin) absorb(x);
    }
    // View.
    F.zoom = num_field(cfg, "zoom", false, 1.0f);
    if (const Json* v = cfg.get("pan_x"); v && v->kind == Json::Number) F.pan_x = v->num;
    if (const Json* v = cfg.get("pan_y"); v && v->kind == Json::Number) F.pan_y = v->num;
    F.rotation = num_field(cfg, "rotation", false, 0.0f);
    // Palette (palette.rs:453-482, 890-910; default Palette::fire, palette.rs:148-174).
    if (const Json* p = cfg.get("palette"); p && p->kind == Json::Object) {
        if (const Json* hx = p->get("indexed_colors"); hx && hx->kind == Json::String) {
            const std::string& s = hx->str;
            size_t i = 0; int k = 0;
            while (i <= s.size()) {
                size_t j = s.find(',', i);
                if (j == std::string::npos) j = s.size();
                std::string h = s.substr(i, j - i);
                if (h.size() != 6) fail("Invalid hex color '" + h + "' at index " + std::to_string(k));
                float rgb[3];
                for (int q = 0; q < 3; ++q) {
                    char* end = nullptr;
                    std::string part = h.substr(q * 2, 2);
                    long v = std::strtol(part.c_str(), &end, 16);
                    if (!end || *end) fail("Invalid hex color '" + h + "'");
                    rgb[q] = (float)v / 255.0f;
                }
                F.stop_pos.push_back((float)k / 255.0f);
                F.stop_col.insert(F.stop_col.end(), rgb, rgb + 3);
                ++k;
                i = j + 1;
            }
        } else if (const Json* st = p->get("stops"); st && st->kind == Json::Array) {
            for (auto& s : st->arr) {
                F.stop_pos.push_back((float)s->number_or("position", 0.0));
                const Json* col = s->get("color");
                for (int q = 0; q < 3; ++q)
                    F.stop_col.push_back(col && col->kind == Json::Array && (int)col->arr.size() > q ? (float)col->arr[q]->num : 1.0f);
            }
        } else fail("a palette with either 'indexed_colors' or 'stops'");
    } else {
        const float pos[5] = {0.0f, 0.25f, 0.5f, 0.75f, 1.0f};
        const float col[15] = {0, 0, 0, 0.5f, 0, 0, 1.0f, 0.3f, 0, 1.0f, 0.8f, 0, 1.0f, 1.0f, 0.8f};
        F.stop_pos.assign(pos, pos + 5);
        F.stop_col.assign(col, col + 15);
    }
    F.palette_size = (int)num_field(cfg, "palette_size", false, 256.0f);
    if (F.palette_size < 2 || F.palette_size > 4096) fail("palette_size must be 2..4096");
    F.palette_rotation = num_field(cfg, "palette_rotation", false, 0.0f);
    F.palette_reverse = cfg.bool_or("palette_reverse", false);
    F.palette_squeeze = num_field(cfg, "palette_squeeze", false, 1.0f);              // fractal_config.rs:436-456
    F.palette_squeeze_falloff = num_field(cfg, "palette_squeeze_falloff", false, 0.5f);
    F.palette_log_strength = num_field(cfg, "palette_log_strength", false, 0.0f);
    if (const Json* m = cfg.get("palette_squeeze_mode"); m && m->kind == Json::String) {
        static const char* const kSqueeze[] = {"linear", "Linear", "geometric", "Geometric"};
        F.palette_squeeze_mode = mode_code(m->str, kSqueeze, 2, "palette squeeze mode");
    }
    if (const Json* cm = cfg.get("color_mode"); cm && cm->kind == Json::String) {
        if (cm->str == "speed" || cm->str == "Speed") F.color_mode = 1;
        else if (cm->str != "Palette" && cm->str != "palette")
            fail("colour mode `" + cm->str + "` is not supported by this build (palette and speed)");
    }
    F.speed_factor = num_field(cfg, "speed_factor", false, 0.5f);      // fractal_config.rs:400-401, 866
    F.filter.radius = num_field(cfg, "filter_radius", false, 0.0f);
    F.filter.blur_edges = num_field(cfg, "filter_blur_edges", false, 0.0f);
    // Tone map (defaults.rs:18-52; fractal_config.rs field defaults).
    ToneMap& tm = F.tm;
    static const char* const kModes[] = {"linear", "Linear", "logarithmic", "Logarithmic", "density", "DensityVisualization"};
    static const char* const kHigh[] = {"clip", "Clip", "max_norm", "MaxNorm", "reinhard", "Reinhard", "filmic", "Filmic", "agx", "AgX", "agx_punchy", "AgXPunchy"};
    if (const Json* m = cfg.get("tonemap_mode"); m && m->kind == Json::String) tm.mode = mode_code(m->str, kModes, 3, "tone map mode");
    if (const Json* m = cfg.get("highlight_mode"); m && m->kind == Json::String) tm.highlight = mode_code(m->str, kHigh, 6, "highlight mode");
    tm.exposure = num_field(cfg, "exposure", false, 1.0f);
    tm.gamma = num_field(cfg, "gamma", false, 4.0f);
    tm.gamma_threshold = num_field(cfg, "gamma_threshold", false, 5.0f);
    tm.brightness = num_field(cfg, "brightness", false, 4.0f);
    tm.vibrancy = num_field(cfg, "vibrancy", false, 1.0f);
    tm.white_level = num_field(cfg, "white_level", false, 200.0f);
    tm.saturation = num_field(cfg, "saturation", false, 1.0f);
    tm.hue_shift = num_field(cfg, "hue_shift", false, 0.0f);
    tm.alpha_blend_low = num_field(cfg, "alpha_blend_low", false, 0.3f);
    tm.alpha_blend_high = num_field(cfg, "alpha_blend_high", false, 0.8f);
    tm.density_scale = num_field(cfg, "density_scale", false, 1.0f);
    tm.levels_enabled = cfg.bool_or("levels_enabled", true);
    tm.levels_low = num_field(cfg, "levels_low", false, 0.0f);
    tm.levels_high = num_field(cfg, "levels_high", false, 10.0f);
    tm.levels_gamma = num_field(cfg, "levels_gamma", false, 0.5f);
    if (const Json* bg = cfg.get("background_color"); bg && bg->kind == Json::Array)
        for (int q = 0; q < 3 && q < (int)bg->arr.size(); ++q) tm.background[q] = (float)bg->arr[q]->num;
    tm.use_curve = cfg.bool_or("use_curve", true);
    if (const Json* tc = cfg.get("tonemap_curve"); tc && tc->kind == Json::Object) {
        if (const Json* pts = tc->get("points"); pts && pts->kind == Json::Array && pts->arr.size() >= 2) {
            tm.curve.clear();
            for (auto& p : pts->arr) tm.curve.push_back({(float)p->number_or("x", 0), (float)p->number_or("y", 0)});
        }
    }
    // Density estimation: this build's extension (flam3's estimator
    // radius / minimum / curve; the reference writes them unused,
    // src/flame_xml.rs:1488-1490).
    if (const Json* de = cfg.get("density_estimation"); de && de->kind == Json::Object) {
        F.de.max_radius = (float)de->number_or("radius", 0.0);
        F.de.min_radius = (float)de->number_or("minimum", 0.0);
        F.de.curve = (float)de->number_or("curve", 0.4);
        if (!(F.de.max_radius >= 0 && F.de.max_radius <= 32)) fail("density_estimation.radius must be 0..32");
        if (!(F.de.min_radius >= 0 && F.de.min_radius <= 32)) fail("density_estimation.minimum must be 0..32");
        if (!(F.de.curve >= 0 && F.de.curve <= 16)) fail("density_estimation.curve must be 0..16");
    }
    if (const Json* mi = cfg.get("max_iterations"); mi && mi->kind == Json::Number) F.max_iterations = (uint64_t)mi->num;
    F.deterministic_rng = cfg.bool_or("deterministic_rng", false);
    if (F.deterministic_rng) F.seed = 12345;
    else {
        std::random_device rd;
        F.seed = ((uint64_t)rd() << 32) | rd();
    }
    return F;
}

Flame parse_config_text(const std::string& text) {
    JsonPtr j;
    try { j = json_parse(text); }
    catch (const std::exception& e) { fail(std::string("config is not JSON: ") + e.what()); }
    return parse_config(*j);
}

// Round-to-nearest-even half precision (the palette and curve texels,
// gpu/buffers.rs:3215-3221, tonemap.rs:289-304).
float f16_round(float v) {
    uint32_t x; std::memcpy(&x, &v, 4);
    uint32_t sign = x & 0x80000000u; x ^= sign;
    float a; std::memcpy(&a, &x, 4);
    float r;
    if (x >= 0x477ff000u) r = 65504.0f;
    else if (x < 0x38800000u) r = std::nearbyint(a * 16777216.0f) / 16777216.0f;
    else {
        uint32_t lsb = (x >> 13) & 1u;
        x += 0xfffu + lsb;
        x &= ~0x1fffu;
        std::memcpy(&r, &x, 4);
    }
    uint32_t rb; std::memcpy(&rb, &r, 4); rb |= sign; std::memcpy(&r, &rb, 4);
    return r;
}

std::vector<float> palette_table(const Flame& f) {
    const int size = f.palette_size;
    const int ns = (int)f.stop_pos.size();
    const float* pos = f.stop_pos.data();
    const float* col = f.stop_col.data();
    std::vector<float> base((size_t)size * 3);
    for (int i = 0; i < size; ++i) {                       // palette.rs:265-278
        float t = (float)i / (float)(size - 1);
        float c[3] = {1.f, 1.f, 1.f};
        if (ns > 0) {                                      // palette.rs:310-360
            t = std::min(std::max(t, 0.f), 1.f);
            if (t < pos[0]) { for (int k = 0; k < 3; ++k) c[k] = col[k]; }
            else {
                int idx = 0;
                for (int s = 0; s < ns; ++s) { if (pos[s] > t) break; idx = s; }
                if (idx == ns - 1) { for (int k = 0; k < 3; ++k) c[k] = col[idx * 3 + k]; }
                else {
                    float range = pos[idx + 1] - pos[idx];
                    if (range < 1e-6f) { for (int k = 0; k < 3; ++k) c[k] = col[idx * 3 + k]; }
                    else {
                        float lt = (t - pos[idx]) / range;
                        for (int k = 0; k < 3; ++k) c[k] = col[idx * 3 + k] + (col[(idx + 1) * 3 + k] - col[idx * 3 + k]) * lt;
                    }
                }
            }
        }
        for (int k = 0; k < 3; ++k) base[(size_t)i * 3 + k] = c[k];
    }
    // Squeeze, then redistribution (palette.rs:703-766): entry i reads the
    // previous table at floor(src_t * size) (saturating, at most size - 1)
    // for src_t the stage's map of t = i / size.
    auto remap = [&](std::vector<float>& tab, const std::function<float(float)>& map) {
        std::vector<float> out((size_t)size * 3);
        for (int i = 0; i < size; ++i) {
            const float src_t = map((float)i / (float)size);
            const float fi = src_t * (float)size;
            const size_t src = std::min<size_t>(!(fi > 0.0f) ? 0 : fi >= 1.8e19f ? SIZE_MAX : (size_t)fi, (size_t)size - 1);
            for (int k = 0; k < 3; ++k) out[(size_t)i * 3 + k] = tab[src * 3 + k];
        }
        tab = out;
    };
    if (f.palette_squeeze_mode == 0 && f.palette_squeeze != 1.0f) {
        const float factor = f.palette_squeeze;
        remap(base, [factor](float t) { const float x = t * factor; return x - std::trunc(x); });
    } else if (f.palette_squeeze_mode == 1) {
        const float r = f.palette_squeeze_falloff;
        remap(base, [r](float t) {                        // geometric_squeeze_lookup, palette.rs:607-640
            if (r >= 0.999f) return t;
            if (r <= 0.001f) return std::min(std::max(t / std::max(r, 1e-6f), 0.0f), 1.0f);
            if (t <= 0.0f) return 0.0f;
            float start = 0.0f, rn = 1.0f;
            for (int n = 0; n < 64; ++n) {
                const float width = rn * (1.0f - r);
                const float end = start + width;
                if (t < end) return width <= 0.0f ? 0.0f : std::min(std::max((t - start) / width, 0.0f), 1.0f);
                start = end;
                rn *= r;
                if (rn < 1e-10f) return 1.0f;
            }
            return 1.0f;
        });
    }
    if (std::fabs(f.palette_log_strength) >= std::numeric_limits<float>::epsilon()) {
        const float s = f.palette_log_strength;
        remap(base, [s](float t) {                        // log_redistribute_lookup, palette.rs:653-671
            if (s > 0.0f) {
                const float d = std::expm1(s);
                return d == 0.0f ? t : std::min(std::max(std::expm1(s * t) / d, 0.0f), 1.0f);
            }
            const float d = std::expm1(-s);
            return d == 0.0f ? t : std::min(std::max(1.0f - std::expm1(-s * (1.0f - t)) / d, 0.0f), 1.0f);
        });
    }
    std::vector<float> rot = base;
    if (f.palette_rotation != 0.f) {                      // palette.rs:768-783
        int amt = (int)std::round(f.palette_rotation * (float)size);
        for (int i = 0; i < size; ++i) {
            int src = ((i + amt) % size + size) % size;
            for (int k = 0; k < 3; ++k) rot[(size_t)i * 3 + k] = base[(size_t)src * 3 + k];
        }
    }
    std::vector<float> out((size_t)size * 4);
    for (int i = 0; i < size; ++i) {
        int src = f.palette_reverse ? size - 1 - i : i;    // palette.rs:786-797
        for (int k = 0; k < 3; ++k) {
            float v = f16_round(std::min(std::max(rot[(size_t)src * 3 + k], 0.f), 1.f));
            out[(size_t)i * 4 + k] = (float)std::pow((double)std::max(v, 0.f), 2.2);   // utilities.wgsl:143-145
        }
        out[(size_t)i * 4 + 3] = 1.0f;
    }
    return out;
}

// ToneCurve::evaluate (src/scene/tonemap.rs:209-284): monotone cubic Hermite.
static float curve_eval(const std::vector<CurvePt>& pts, float x) {
    x = std::min(std::max(x, 0.0f), 1.0f);
    for (size_t i = 0; i + 1 < pts.size(); ++i) {
        const CurvePt& p0 = pts[i];
        const CurvePt& p1 = pts[i + 1];
        if (x >= p0.x && x <= p1.x) {
            float delta = (p1.y - p0.y) / (p1.x - p0.x);
            float m0 = i == 0 ? delta : ((p0.y - pts[i - 1].y) / (p0.x - pts[i - 1].x) + delta) * 0.5f;
            float m1 = i == pts.size() - 2 ? delta : (delta + (pts[i + 2].y - p1.y) / (pts[i + 2].x - p1.x)) * 0.5f;
            float m0f, m1f;
            if (std::fabs(delta) < 1e-6f) { m0f = 0; m1f = 0; }
            else {
                float al = m0 / delta, be = m1 / delta;
                if (al < 0 || be < 0) { m0f = delta; m1f = delta; }
                else {
                    float ss = al * al + be * be;
                    if (ss > 9.0f) { float tau = 3.0f / std::sqrt(ss); m0f = tau * al * delta; m1f = tau * be * delta; }
                    else { m0f = m0; m1f = m1; }
                }
            }
            float t = (x - p0.x) / (p1.x - p0.x);
            float t2 = t * t, t3 = t2 * t;
            float h00 = 2.0f * t3 - 3.0f * t2 + 1.0f, h10 = t3 - 2.0f * t2 + t;
            float h01 = -2.0f * t3 + 3.0f * t2, h11 = t3 - t2;
            float dx = p1.x - p0.x;
            return h00 * p0.y + h10 * dx * m0f + h01 * p1.y + h11 * dx * m1f;
        }
    }
    return x;
}

std::vector<float> curve_lut(const ToneMap& tm) {
    std::vector<float> lut(256);
    for (int i = 0; i < 256; ++i) lut[i] = f16_round(curve_eval(tm.curve, (float)i / 255.0f));
    return lut;
}

}  // namespace ffb
