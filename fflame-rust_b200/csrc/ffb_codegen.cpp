// ffb_codegen.cpp -- see ffb_codegen.hpp.

#include "ffb_codegen.hpp"

#include <algorithm>
#include <cmath>
#include <functional>
#include <sstream>
#include <stdexcept>

#include "ffb_device_src.inc"

namespace ffb {

namespace {

constexpr int kSymBlock = 6 + 64;            // post-symmetry table block (floats)
constexpr int kMaxDrawSlots = 64;            // draws an iteration (pick, opacity, variations)

// Normal-phase variations: those a normal transform uses at a weight other
// than 0, in local order.  The reference emits every active variation and
// gates each on `xform.variations[idx] != 0.0` (shader_builder_v2.rs
// 2755-2763); one no transform uses never fires, so leaving it out changes
// nothing.
std::vector<const VarDef*> normal_vars(const Flame& f) {
    std::vector<const VarDef*> out;
    for (const VarDef* v : f.local) {
        bool used = false;
        for (auto& x : f.xf) used |= x.var_weight(v) != 0.0f;
        if (used) out.push_back(v);
    }
    return out;
}

std::vector<const VarDef*> final_vars(const Flame& f, const XForm& x) {
    std::vector<const VarDef*> out;
    for (const VarDef* v : f.local) if (x.var_weight(v) != 0.0f) out.push_back(v);
    return out;
}

// Where one call of a variation finds its inputs, as source expressions:
// its packed parameter row (`prm(q)`), its own weight and its transform's
// affine (`xf(0..5)` = a..f), and the first of its draw slots.
struct Site {
    std::function<std::string(int)> prm;
    std::string w;
    std::function<std::string(int)> xf;
    int slot = -1;
    std::string st;     // stateful variations: the walker's first state slot of this call (float*)
    std::string inst;   // subflames: the instance number keying the subflame's own stream (u32)
};

// The walker's state slots (compute_state_layout, transforms.rs:226-300):
// transform by transform in the reference's xform-id order -- normals, the
// final pool, then each subflame's normals and finals -- the stateful
// variations it uses, in local order.  A subflame variation inside a
// subflame never runs (the inner dispatcher leaves it out) and takes none.
// `init` marks the entries whose `wgsl_state_init` runs each dispatch (the
// reference's layout holds weights above 1e-6 in magnitude).
struct StEntry {
    int kind;               // 0 normal, 3 linked, 1 final (pool indices), 2 subflame s, transform t (normals then finals)
    int s, t;
    const VarDef* v;
    int base;
    bool init;
};

std::vector<StEntry> state_layout(const Flame& f, int& total) {
    std::vector<StEntry> out;
    int cur = 0;
    auto lid = [&](const VarDef* v) { return (int)(std::find(f.local.begin(), f.local.end(), v) - f.local.begin()); };
    auto emit = [&](int kind, int sidx, int t, const XForm& x) {
        std::vector<std::pair<const VarDef*, float>> vs;
        for (auto& pv : x.vars)
            if (pv.second != 0.0f && pv.first->state > 0 && !(kind == 2 && (pv.first->flags & VF_SUB))) vs.push_back(pv);
        std::sort(vs.begin(), vs.end(), [&](const auto& a, const auto& b) { return lid(a.first) < lid(b.first); });
        for (auto& pv : vs) {
            out.push_back({kind, sidx, t, pv.first, cur, pv.first->init_draws > 0 && std::fabs(pv.second) > 1e-6f});
            cur += pv.first->state;
        }
    };
    for (size_t k = 0; k < f.xf.size(); ++k) emit(0, 0, (int)k, f.xf[k]);
    for (size_t c = 0; c < f.lnk.size(); ++c) emit(3, 0, (int)c, f.lnk[c]);
    for (size_t c = 0; c < f.fin.size(); ++c) emit(1, 0, (int)c, f.fin[c]);
    for (size_t si = 0; si < f.sub.size(); ++si) {
        const SubFlame& S = f.sub[si];
        for (size_t t = 0; t < S.xf.size() + S.fin.size(); ++t)
            emit(2, (int)si, (int)t, t < S.xf.size() ? S.xf[t] : S.fin[t - S.xf.size()]);
    }
    total = cur;
    return out;
}

int state_base(const std::vector<StEntry>& L, int kind, int sidx, int t, const VarDef* v) {
    for (auto& e : L) if (e.kind == kind && e.s == sidx && e.t == t && e.v == v) return e.base;
    return -1;
}

// A subflame's inner transforms (normals then finals) and, per transform,
// the variations its dispatcher runs: weight other than 0, no subflame
// variation (shader_builder_v2.rs:2391-2420), local order.
std::vector<const VarDef*> inner_vars(const Flame& f, const XForm& x) {
    std::vector<const VarDef*> out;
    for (const VarDef* v : f.local)
        if (!(v->flags & VF_SUB) && x.var_weight(v) != 0.0f) out.push_back(v);
    return out;
}
const XForm& inner_xf(const SubFlame& S, size_t t) { return t < S.xf.size() ? S.xf[t] : S.fin[t - S.xf.size()]; }

// Inner transform record: affine a..f, post a..f, post flag, colour
// C1, C2, opacity, direct colour, then per variation its weight, its
// packed parameters and (stateful) its state base.
constexpr int kSubRec = 17;
int inner_rec_size(const std::vector<const VarDef*>& vs) {
    int n = kSubRec;
    for (const VarDef* v : vs) n += 1 + v->slots() + (v->state > 0 ? 1 : 0);
    return n;
}

// Normal transform k's site (k a source expression).
Site normal_site(const Plan& p, int j, const std::string& k) {
    Site c;
    const int off = p.vp_off[j];
    c.prm = [off, k](int q) { return "sm[T_VP + " + std::to_string(off + q) + " * FFB_MAXX + " + k + "]"; };
    c.w = "sm[T_VW + " + std::to_string(j) + " * FFB_MAXX + " + k + "]";
    c.xf = [k](int f) { return "sm[T_XF + " + std::to_string(f) + " * FFB_MAXX + " + k + "]"; };
    c.slot = p.normal_slot[j];
    if (p.st_row[j] >= 0) {
        const std::string b = "sm[T_ST + " + std::to_string(p.st_row[j]) + " * FFB_MAXX + " + k + "]";
        c.st = "ffb_st(ctx, " + b + ")";
        c.inst = "ffb_u32(" + b + ")";
    }
    return c;
}

// Final c's site: its record q (affine at q[0..5], weights at q[13..],
// then the parameter rows, then each variation's state base).
Site final_site(const Plan::Fin& fi, int j) {
    Site c;
    const int nv = (int)fi.vars.size(), off = 13 + nv + fi.prm_off[j];
    c.prm = [off](int q) { return "q[" + std::to_string(off + q) + "]"; };
    c.w = "q[" + std::to_string(13 + j) + "]";
    c.xf = [](int f) { return "q[" + std::to_string(f) + "]"; };
    c.slot = fi.slot[j];
    const std::string b = "q[" + std::to_string(13 + nv + fi.prm_slots + j) + "]";
    c.st = "ffb_st(ctx, " + b + ")";
    c.inst = "ffb_u32(" + b + ")";
    return c;
}

// Inner variation j of a subflame transform whose record is q.
Site inner_site(const std::vector<const VarDef*>& vs, int j) {
    int off = kSubRec;
    for (int i = 0; i < j; ++i) off += 1 + vs[i]->slots() + (vs[i]->state > 0 ? 1 : 0);
    Site c;
    c.w = "q[" + std::to_string(off) + "]";
    c.prm = [off](int q) { return "q[" + std::to_string(off + 1 + q) + "]"; };
    c.xf = [](int f) { return "q[" + std::to_string(f) + "]"; };
    c.slot = 0;                                   // the subflame's draws are sequential
    if (vs[j]->state > 0) c.st = "ffb_st(ctx, q[" + std::to_string(off + 1 + vs[j]->slots()) + "])";
    return c;
}

void emit_phases(std::ostringstream& s, const std::vector<const VarDef*>& vars, const std::function<Site(int)>& site,
                 const char* ind, bool gate, const char* vc = "ctx.vc");

// One subflame (subflame.wgsl:254-412, 2-D arm): from the walker's state
// (point, colour, last output; a zero point or a non-finite one walks the
// 42-step prefuse from a random start), step the inner chaos game until a
// visible transform (opacity 1, or its roll passes; at most 1000 steps past
// the prefuse), map the point through the finals to q, place q by scale,
// rotation and offset, and keep the walk and q in the state.  State slots:
// x, y, colour, q.x, q.y, q.colour.  Inner transform t's record at
// sm[rec[t]]; the block at sm[blk]: total weight (at least 1e-6), whether
// any transform can be visible, the running sums of the weights.
void emit_subflame(std::ostringstream& s, const Flame& f, int si, int blk, const std::vector<int>& rec) {
    const SubFlame& S = f.sub[si];
    const int N = (int)S.xf.size();
    s << "template <class S> __device__ void ffb_sub_" << si << "(const float* __restrict__ sm, FfbCtx& ctx, S& rng, float scale, "
         "float cs, float sn, float offx, float offy, float* st, float& qx, float& qy, float& qw) {\n";
    if (N == 0) {
        s << "    (void)sm; (void)ctx; (void)rng; (void)scale; (void)cs; (void)sn; (void)offx; (void)offy; (void)st;\n"
             "    qx = 0.0f; qy = 0.0f; qw = 0.0f;\n}\n";
        return;
    }
    s << "    const u32 sd = ctx.stride;\n"
         "    float px = st[0], py = st[sd], color = st[2 * sd];\n"
         "    const bool pre = (px == 0.0f && py == 0.0f) || !(fabsf(px) <= 1e32f) || !(fabsf(py) <= 1e32f) || !(fabsf(color) <= 1e32f);\n"
         "    if (pre) { px = rng.draw(0) - 0.5f; py = rng.draw(0) - 0.5f; color = rng.draw(0); }\n"
         "    const float* B = sm + " << blk << ";\n"
         "    const u32 pre_steps = pre ? 42u : 0u;\n"
         "    const u32 steps = pre_steps + (B[1] > 0.5f ? 1000u : 0u);\n"
         "    bool visible = false;\n"
         "    for (u32 it = 0; it < steps; ++it) {\n"
         "        const float r = rng.draw(0) * B[0];\n"
         "        int pk = " << N - 1 << ";\n"
         "        for (int i = 0; i < " << N << "; ++i) if (r < B[2 + i]) { pk = i; break; }\n"
         "        float op = 1.0f;\n"
         "        switch (pk) {\n";
    auto body = [&](size_t t, const char* pin_x, const char* pin_y, const char* cin, const char* pout_x, const char* pout_y,
                    const char* cout, const char* ind) {
        const std::vector<const VarDef*> vs = inner_vars(f, inner_xf(S, t));
        s << ind << "const float* q = sm + " << rec[t] << ";\n"
          << ind << "const float cb = " << cin << " * q[13] + q[14];\n"
          << ind << "float vc = cb;\n"
          << ind << "float x = q[0] * " << pin_x << " + q[1] * " << pin_y << " + q[4];\n"
          << ind << "float y = q[2] * " << pin_x << " + q[3] * " << pin_y << " + q[5];\n"
          << ind << "{\n";
        const std::string ind2 = std::string(ind) + "    ";
        emit_phases(s, vs, [&](int j) { return inner_site(vs, j); }, ind2.c_str(), true, "vc");
        s << ind2 << "x = rx; y = ry;\n" << ind << "}\n"
          << ind << "if (q[12] > 0.5f) { const float ux = q[6] * x + q[7] * y + q[10]; const float uy = q[8] * x + q[9] * y + q[11]; x = ux; y = uy; }\n"
          << ind << pout_x << " = x; " << pout_y << " = y; " << cout << " = cb + q[16] * (vc - cb);\n";
    };
    for (int t = 0; t < N; ++t) {
        s << "        case " << t << ": {\n";
        body((size_t)t, "px", "py", "color", "px", "py", "color", "            ");
        s << "            op = q[15];\n            break; }\n";
    }
    s << "        default: break;\n        }\n"
         "        if (it >= pre_steps && (op >= 1.0f || rng.draw(0) < op)) { visible = true; break; }\n"
         "    }\n"
         "    st[0] = px; st[sd] = py; st[2 * sd] = color;\n"
         "    if (!visible) { qx = st[3 * sd]; qy = st[4 * sd]; qw = st[5 * sd]; return; }\n"
         "    float fx = px, fy = py, fc = color;\n";
    for (size_t t = (size_t)N; t < S.xf.size() + S.fin.size(); ++t) {
        s << "    {\n";
        body(t, "fx", "fy", "fc", "fx", "fy", "fc", "        ");
        s << "    }\n";
    }
    s << "    const float x = scale * fx, y = scale * fy;\n"
         "    qx = x * cs - y * sn + offx;\n"
         "    qy = x * sn + y * cs + offy;\n"
         "    qw = fc;\n"
         "    st[3 * sd] = qx; st[4 * sd] = qy; st[5 * sd] = qw;\n}\n";
}

// `v_name(px, py[, rng, slot][, params...][, w][, a..f][, state, stride][, hide], ox, oy)`.
std::string call(const VarDef* v, const Site& c, const char* px = "x", const char* py = "y") {
    std::ostringstream o;
    o << v->fn << "(" << px << ", " << py;
    if (v->draws) o << ", rng, " << c.slot;
    for (int q = 0; q < v->slots(); ++q) o << ", " << c.prm(q);
    if (v->flags & VF_W) o << ", " << c.w;
    if (v->flags & VF_XF) for (int f = 0; f < 6; ++f) o << ", " << c.xf(f);
    if (v->state > 0) o << ", " << c.st << ", ctx.stride";
    if (v->flags & VF_HIDE) o << ", ctx.hide";
    o << ", ox, oy)";
    return o.str();
}

// subflame_wf / pre_subflame_wf (subflame.rs:122-143, 195-204): step the
// subflame (subflame_iterate, placed by scale, angle and offsets), take its
// colour when color_mode is not -1, and return q / weight (the normal
// phase multiplies the weight back) or, in the pre phase, q itself.
// Parameter row: subflame_id, scale, angle, offset_x, offset_y, offset_z,
// colorscale_z, color_mode, cos(angle), sin(angle).
std::string call_sub(const VarDef* v, const Site& c, const char* vc) {
    std::ostringstream o;
    o << "auto&& sq = ffb_sub_stream(rng, ctx, " << c.inst << "); float qx, qy, qw; "
      << "ffb_subflame(sm, ctx, sq, ffb_u32(" << c.prm(0) << "), " << c.prm(1) << ", " << c.prm(8) << ", " << c.prm(9) << ", "
      << c.prm(3) << ", " << c.prm(4) << ", " << c.st << ", qx, qy, qw); "
      << "if (ffb_i32(" << c.prm(7) << ") != -1) " << vc << " = qw; ";
    if (v->flags & VF_PRE) o << "ox = qx; oy = qy;";
    else o << "ox = qx / w; oy = qy / w;";
    return o.str();
}

// The Jacobian of a variation body (ffb_diff_jac.cuh): "v_name" -> "dj_name".
// Only variations flagged VF_JAC have one; they take at most one draw.
std::string jcall(const VarDef* v, const Site& c) {
    std::ostringstream o;
    o << "dj_" << (v->fn + 2) << "(x, y";
    if (v->draws) o << ", rng.draw(" << c.slot << ")";
    for (int q = 0; q < v->slots(); ++q) o << ", " << c.prm(q);
    o << ")";
    return o.str();
}

// The three phases of apply_variations (shader_builder_v2.rs:2589-2800):
// Pre variations replace the input point in turn (`temp = V(temp)`), the
// others sum `w * V(temp)` from zero, Post variations replace the sum
// (`result = V(result)`); each gated on its weight, in local order within
// its phase.  `site(j)` locates variation j of `vars`; `gate` false drops
// the weight test (the per-transform form lists only the variations the
// transform uses).
// `vc` names the colour register a WritesColor variation writes.
void emit_phases(std::ostringstream& s, const std::vector<const VarDef*>& vars,
                 const std::function<Site(int)>& site, const char* ind, bool gate, const char* vc) {
    s << ind << "float tx = x, ty = y, rx = 0.0f, ry = 0.0f, ox, oy;\n";
    auto open = [&](const Site& c) {
        s << ind << "{ const float w = " << c.w << "; " << (gate ? "if (w != 0.0f) { " : "{ ");
    };
    // Passes: Pre, the accumulating normal variations, the Replace ones
    // (shader_builder_v2.rs:2511-2520, 2700-2709: after the others, each
    // assigning `result = w * V(p)` over the sum so far), Post.
    for (int pass = 0; pass < 4; ++pass) {
        for (size_t j = 0; j < vars.size(); ++j) {
            const VarDef* v = vars[j];
            const int ph = (v->flags & VF_PRE) ? 0 : (v->flags & VF_POST) ? 3 : (v->flags & VF_REPLACE) ? 2 : 1;
            if (ph != pass) continue;
            const Site c = site((int)j);
            open(c);
            const std::string body = (v->flags & VF_SUB) ? call_sub(v, c, vc) : call(v, c, ph == 3 ? "rx" : "tx", ph == 3 ? "ry" : "ty") + ";";
            if (ph == 0) s << body << " tx = ox; ty = oy;";
            else if (ph == 1) s << body << " rx = rx + w * ox; ry = ry + w * oy;";
            else if (ph == 2) s << body << " rx = w * ox; ry = w * oy;";
            else s << body << " rx = ox; ry = oy;";
            s << " } }   // " << v->name << "\n";
        }
    }
}

// The differentiable render's generated functions and kernels.
void emit_diff(std::ostringstream& s, const Plan& p) {
    const int NVN = (int)p.normal.size();
    s << kDiffJacSrc << "\n";
    s << "#define FFB_WINDOW " << p.diff_window << "\n#define FFB_CKPT " << p.diff_ckpt << "\n";
    s << "#define FFB_NPARAM " << p.maxx * (7 + NVN) << "\n";
    // Normal phase of transform k for the adjoint: the weight gradient of
    // each variation (a . V_j(x, y)) into gw[j * P], and J = sum_j w_j J_j.
    s << "template <class R> __device__ __forceinline__ void ffb_dnormal(const float* __restrict__ sm, int k, float x, float y, R& rng, "
         "float ax, float ay, float* __restrict__ gw, int P, float4& J) {\n";
    s << "    J = make_float4(0.f, 0.f, 0.f, 0.f);\n    float ox, oy;\n";
    for (int j = 0; j < NVN; ++j) {
        const VarDef* v = p.normal[j];
        const Site c = normal_site(p, j, "k");
        s << "    { " << call(v, c) << "; const float g = ax * ox + ay * oy; if (isfinite(g)) gw["
          << j << " * P] += g;\n      const float w = " << c.w << "; if (w != 0.0f) { const float4 jj = "
          << jcall(v, c) << "; J.x += w * jj.x; J.y += w * jj.y; J.z += w * jj.z; J.w += w * jj.w; } }   // " << v->name << "\n";
    }
    s << "    if (!(isfinite(J.x) && isfinite(J.y) && isfinite(J.z) && isfinite(J.w))) J = make_float4(0.f, 0.f, 0.f, 0.f);\n}\n";
    // One normal variation's value and Jacobian (the probe).
    s << "template <class R> __device__ __forceinline__ void ffb_dvar_one(const float* __restrict__ sm, int j, int k, float x, float y, R& rng, "
         "float& ox, float& oy, float4& J) {\n    switch (j) {\n";
    for (int j = 0; j < NVN; ++j) {
        const VarDef* v = p.normal[j];
        const Site c = normal_site(p, j, "k");
        s << "    case " << j << ": " << call(v, c) << "; J = " << jcall(v, c) << "; break;\n";
    }
    s << "    default: ox = 0.f; oy = 0.f; J = make_float4(0.f, 0.f, 0.f, 0.f); break;\n    }\n}\n";
    s << kDiffSrc << "\n";
}

std::string jac_names() {
    std::string o;
    for (const VarDef* v : registry_all()) if (v->flags & VF_JAC) o += (o.empty() ? "" : ", ") + std::string(v->name);
    return o;
}

}  // namespace

Plan make_plan(const Flame& f, int rng_mode, int math_mode, int maxx, int threads, bool per_xform, bool exact,
               int diff_window, int diff_ckpt, bool emit, bool defer) {
    Plan p;
    p.exact = exact;
    p.emit = emit;
    p.defer = defer && !emit && diff_window == 0;
    p.diff_window = diff_window;
    p.diff_ckpt = diff_ckpt;
    p.rng_mode = rng_mode;
    p.math_mode = math_mode;
    p.per_xform = per_xform;
    p.threads = threads;
    p.maxx = std::max<int>(maxx, (int)f.xf.size());
    p.normal = normal_vars(f);
    // Draw slots: 0 the transform pick, 1 the opacity test, then each
    // NeedsRng variation's draws (consecutive, in its body's order): the
    // normal phase's in local order, then each attached linked transform's,
    // then each attached final's.
    int slot = 2, vp = 0;
    for (const VarDef* v : p.normal) {
        p.normal_slot.push_back(v->draws ? slot : -1);
        slot += v->draws;
        p.vp_off.push_back(vp);
        vp += v->slots();
    }
    p.vp_slots = vp;
    auto chain_entry = [&](const XForm& x) {
        Plan::Fin fi;
        fi.vars = final_vars(f, x);
        int fo = 0;
        for (const VarDef* v : fi.vars) {
            fi.slot.push_back(v->draws ? slot : -1);
            slot += v->draws;
            fi.prm_off.push_back(fo);
            fo += v->slots();
        }
        fi.prm_slots = fo;
        return fi;
    };
    for (int c : f.lnk_used) { p.lnk.push_back(chain_entry(f.lnk[c])); p.lnk_pool.push_back(c); }
    p.fin_slot0 = slot;
    for (int c : f.fin_used) { p.fin.push_back(chain_entry(f.fin[c])); p.fin_pool.push_back(c); }
    p.n_slots = slot;
    auto index_of = [](const std::vector<int>& pool, int c) { return (int)(std::find(pool.begin(), pool.end(), c) - pool.begin()); };
    p.fin_uniform = f.fin_uniform;
    if (p.fin_uniform) for (int c : f.fin_chain) p.fin_chain.push_back(index_of(p.fin_pool, c));
    for (auto& x : f.xf) {
        p.lcap = std::max(p.lcap, (int)x.linked_att.size());
        if (!p.fin_uniform) p.fcap = std::max(p.fcap, (int)x.final_att.size());
        // With the counter-based stream a transform's draws have fixed
        // slots: one chain running a drawing transform twice would draw the
        // same words twice.
        if (rng_mode == RNG_PHILOX) {
            auto repeats = [&](const std::vector<int>& att, const std::vector<XForm>& pool) {
                for (size_t i = 0; i < att.size(); ++i)
                    for (size_t j = i + 1; j < att.size(); ++j)
                        if (att[i] == att[j])
                            for (const VarDef* v : final_vars(f, pool[(size_t)att[i]]))
                                if (v->draws) return true;
                return false;
            };
            if (repeats(x.linked_att, f.lnk) || repeats(x.final_att, f.fin))
                throw std::runtime_error("a chain attaching the same randomised transform twice needs the pcg stream in this build");
        }
    }
    int n_state = 0;
    const std::vector<StEntry> layout = state_layout(f, n_state);
    p.n_state = n_state;
    for (auto& e : layout) p.n_init += e.init ? 1 : 0;
    // Speed colour: three more slots a walker; its colour travels with the
    // walker, so the plot stays inline and the splat unaggregated.
    p.speed = f.color_mode == 1;
    if (p.speed) {
        p.speed_slot = p.n_state;
        p.n_state += 3;
        p.defer = false;
    }
    p.st_row.assign(p.normal.size(), -1);
    int st_rows = 0;
    for (size_t j = 0; j < p.normal.size(); ++j) {
        if (p.normal[j]->state > 0) p.st_row[j] = st_rows++;
        p.dc |= (p.normal[j]->flags & VF_DC) != 0;
        p.hide |= (p.normal[j]->flags & VF_HIDE) != 0;
    }
    for (const auto* list : {&p.lnk, &p.fin})
        for (auto& fi : *list)
            for (const VarDef* v : fi.vars) p.hide |= (v->flags & VF_HIDE) != 0;
    // The deferred plot runs the finals out of walker order, with the draws
    // captured at their static slots: finals that carry state or step a
    // subflame stay inline.
    for (auto& fi : p.fin)
        for (const VarDef* v : fi.vars)
            if (v->state > 0 || (v->flags & VF_SUB)) p.defer = false;
    // A subflame call's own stream holds 2^18 words an instance.
    for (const SubFlame& S : f.sub) {
        int most = 0, fin = 0;
        for (size_t t = 0; t < S.xf.size() + S.fin.size(); ++t) {
            int d = 0;
            for (const VarDef* v : inner_vars(f, inner_xf(S, t))) d += v->draws;
            if (t < S.xf.size()) most = std::max(most, d); else fin += d;
        }
        if (3 + 1042 * (2 + most) + fin >= (1 << 18))
            throw std::runtime_error("a subflame's transforms take too many random draws a step for this build");
    }
    // Philox words live in registers (4 a block): a bound keeps them there.
    if (p.n_slots > kMaxDrawSlots)
        throw std::runtime_error("the flame's variations take " + std::to_string(p.n_slots - 2) +
                                 " random draws an iteration, over the " + std::to_string(kMaxDrawSlots - 2) + " this build carries");
    if (diff_window > 0) {
        // The adjoint differentiates the weighted sum through each
        // variation's Jacobian; a variation without one (or outside the
        // normal phase) cannot be differentiated here.
        auto need = [](const VarDef* v) {
            if (!(v->flags & VF_JAC))
                throw std::runtime_error("variation `" + std::string(v->name) +
                                         "` has no Jacobian in this build; the differentiable render supports " + jac_names());
        };
        for (const VarDef* v : p.normal) need(v);
        for (auto& fi : p.fin) for (const VarDef* v : fi.vars) need(v);
        if (!f.xaos.empty()) throw std::runtime_error("the differentiable render has no xaos");
    }
    for (auto& x : f.xf) p.has_post |= x.post;
    const int M = p.maxx, NVN = (int)p.normal.size();
    constexpr int kXfFields = 17;                 // F_NFIELDS of ffb_device.cuh
    p.t_cum = 1;
    p.t_xf = p.t_cum + M;
    p.t_vw = p.t_xf + kXfFields * M;
    p.t_vp = p.t_vw + NVN * M;
    p.t_fin = p.t_vp + p.vp_slots * M;
    int off = p.t_fin;
    for (auto& fi : p.fin) { fi.off = off; off += 13 + 2 * (int)fi.vars.size() + fi.prm_slots; }
    for (auto& li : p.lnk) { li.off = off; off += 13 + 2 * (int)li.vars.size() + li.prm_slots; }
    p.t_att = off;
    if (p.lcap > 0 || p.fcap > 0) off += M * (2 + p.lcap + p.fcap);
    p.sym_kind = f.sym.kind;
    p.t_sym = off;
    if (p.sym_kind != 0) off += kSymBlock;
    p.xaos = !f.xaos.empty();
    p.t_xaos = off;
    if (p.xaos) off += M * (M + 1);
    p.t_speed = off;
    if (p.speed) off += 1;
    p.t_st = off;
    off += st_rows * M;
    p.t_init = off;
    off += p.n_init;
    for (const SubFlame& S : f.sub) {
        p.sub_blk.push_back(off);
        off += 2 + (int)S.xf.size();
        std::vector<int> rec;
        for (size_t t = 0; t < S.xf.size() + S.fin.size(); ++t) {
            rec.push_back(off);
            off += inner_rec_size(inner_vars(f, inner_xf(S, t)));
        }
        p.sub_rec.push_back(rec);
    }
    p.table_size = off;

    std::ostringstream s;
    s << "// generated by ffb_codegen for one flame structure\n";
    s << "#define FFB_MAXX " << M << "\n#define FFB_NVN " << NVN << "\n#define FFB_NFIN " << p.fin.size() << "\n";
    s << "#define FFB_NLNK " << p.lnk.size() << "\n#define FFB_LCAP " << p.lcap << "\n#define FFB_FCAP " << p.fcap
      << "\n#define FFB_ATT_STRIDE " << (2 + p.lcap + p.fcap) << "\n#define T_ATT " << p.t_att << "\n#define FFB_FIN_SLOT0 "
      << p.fin_slot0 << "\n";
    s << "#define FFB_HAS_POST " << (p.has_post ? 1 : 0) << "\n#define FFB_NSLOTS " << p.n_slots << "\n";
    s << "#define FFB_RNG_MODE " << rng_mode << "\n#define FFB_THREADS " << threads << "\n";
    if (math_mode == MATH_SFU) s << "#define FFB_SFU 1\n";
    if (exact) s << "#define FFB_EXACT 1\n";
    if (emit) s << "#define FFB_EMIT 1\n";
    int nfd = 0;
    for (auto& fi : p.fin) for (const VarDef* v : fi.vars) nfd += v->draws;
    if (p.defer) s << "#define FFB_DEFER 1\n#define FFB_NFD " << nfd << "\n";
    s << "#define FFB_SYM_KIND " << p.sym_kind << "\n#define T_SYM " << p.t_sym << "\n";
    if (p.xaos) s << "#define FFB_XAOS 1\n#define T_XAOS " << p.t_xaos << "\n";
    if (f.orbit_refresh) s << "#define FFB_REFRESH " << f.orbit_refresh << "\n";
    s << "#define FFB_NSTATE " << p.n_state << "\n#define FFB_NINIT " << p.n_init << "\n#define T_ST " << p.t_st
      << "\n#define T_INIT " << p.t_init << "\n";
    if (p.dc) s << "#define FFB_DC 1\n";
    if (p.hide) s << "#define FFB_HIDE 1\n";
    if (p.speed) s << "#define FFB_SPEED 1\n#define FFB_SPEED_SLOT " << p.speed_slot << "\n#define T_SPEED " << p.t_speed << "\n";
    s << "#define FFB_TABLE_SIZE " << p.table_size << "\n#define FFB_TABLE_VEC4 " << (p.table_size + 3) / 4 << "\n";
    s << "#define T_TOTAL 0\n#define T_CUM " << p.t_cum << "\n#define T_XF " << p.t_xf << "\n#define T_VW " << p.t_vw
      << "\n#define T_VP " << p.t_vp << "\n";
    s << kDeviceSrc << "\n";
    // Subflames, and the step of subflame `id` (an id with no subflame
    // behind it returns 0 and keeps no state, as an empty subflame does).
    for (size_t si = 0; si < f.sub.size(); ++si) emit_subflame(s, f, (int)si, p.sub_blk[si], p.sub_rec[si]);
    s << "template <class S> __device__ __forceinline__ void ffb_subflame(const float* __restrict__ sm, FfbCtx& ctx, S& rng, u32 id, "
         "float scale, float cs, float sn, float offx, float offy, float* st, float& qx, float& qy, float& qw) {\n    switch (id) {\n";
    for (size_t si = 0; si < f.sub.size(); ++si)
        s << "    case " << si << ": ffb_sub_" << si << "(sm, ctx, rng, scale, cs, sn, offx, offy, st, qx, qy, qw); return;\n";
    s << "    default: (void)sm; (void)ctx; (void)rng; (void)scale; (void)cs; (void)sn; (void)offx; (void)offy; (void)st;\n"
         "        qx = 0.0f; qy = 0.0f; qw = 0.0f; return;\n    }\n}\n";
    // The normal phase (shader_builder_v2.rs:2714-2795): `result += w * V(p)`
    // from zero, in local order, each gated on its weight.
    s << "template <class R> __device__ __forceinline__ void ffb_normal(const float* __restrict__ sm, int k, float& x, float& y, R& rng, FfbCtx& ctx) {\n";
    emit_phases(s, p.normal, [&](int j) { return normal_site(p, j, "k"); }, "    ", true);
    s << "    x = rx; y = ry; (void)ctx;\n}\n";
    // Without a walker (the differentiable render, which has no stateful variations).
    s << "template <class R> __device__ __forceinline__ void ffb_normal(const float* __restrict__ sm, int k, float& x, float& y, R& rng) {\n"
         "    FfbCtx ctx{nullptr, 0u, 0.0f, 0u, 0u, 0u, 0ull};\n    ffb_normal(sm, k, x, y, rng, ctx);\n}\n";
    // Per-transform form for the sorted schedule, where k is (mostly)
    // warp-uniform: each case evaluates only its transform's variations, in
    // the same local order, straight-line (their chains overlap).
    s << "template <class R> __device__ __forceinline__ void ffb_normal_k(const float* __restrict__ sm, int k, float& x, float& y, R& rng, FfbCtx& ctx) {\n";
    if (per_xform) {
        s << "    switch (k) {\n";
        for (size_t k = 0; k < f.xf.size(); ++k) {
            s << "    case " << k << ": {\n";
            std::vector<const VarDef*> used;
            std::vector<int> idx;
            for (int j = 0; j < NVN; ++j)
                if (f.xf[k].var_weight(p.normal[j]) != 0.0f) { used.push_back(p.normal[j]); idx.push_back(j); }
            emit_phases(s, used, [&](int u) { return normal_site(p, idx[u], std::to_string(k)); }, "        ", false);
            s << "        x = rx; y = ry;\n        return; }\n";
        }
        s << "    default: ffb_normal(sm, k, x, y, rng, ctx); return;\n    }\n";
    } else {
        s << "    ffb_normal(sm, k, x, y, rng, ctx);\n";
    }
    s << "}\n";
    // One final of the chain (main_template.wgsl:679-704): affine,
    // variations, post-affine; `aff` false evaluates the variations alone.
    // A final's colour writes are dropped (main_template.wgsl:299-300); a
    // linked transform's reach the register (main_template.wgsl:320-326).
    auto emit_chain_one = [&](const char* name, const std::vector<Plan::Fin>& list, const char* vc) {
        s << "template <class R> __device__ __forceinline__ void " << name
          << "(const float* __restrict__ sm, int c, float& x, float& y, R& rng, FfbCtx& ctx, bool aff) {\n";
        s << "    float vcd = 0.0f;\n    (void)vcd; (void)ctx;\n";
        s << "    switch (c) {\n";
        for (size_t c = 0; c < list.size(); ++c) {
            const Plan::Fin& fi = list[c];
            s << "    case " << c << ": {\n        const float* q = sm + " << fi.off << ";\n";
            s << "        if (aff) { float ax = q[0] * x + q[1] * y + q[4]; float ay = q[2] * x + q[3] * y + q[5]; x = ax; y = ay; }\n";
            emit_phases(s, fi.vars, [&](int j) { return final_site(fi, j); }, "        ", true, vc);
            s << "        if (aff && q[12] > 0.5f) { float px = q[6] * rx + q[7] * ry + q[10]; float py = q[8] * rx + q[9] * ry + q[11]; rx = px; ry = py; }\n";
            s << "        x = rx; y = ry;\n        break; }\n";
        }
        s << "    default: break;\n    }\n}\n";
    };
    emit_chain_one("ffb_final_one", p.fin, "vcd");
    emit_chain_one("ffb_linked_one", p.lnk, "ctx.vc");
    // Normal transform k's linked chain, each output feeding the next
    // (main_template.wgsl:320-360), from the attachment table.
    s << "template <class R> __device__ __forceinline__ void ffb_linked(const float* __restrict__ sm, int k, float& x, float& y, R& rng, FfbCtx& ctx) {\n";
    if (!p.lnk.empty())
        s << "    const float* a = sm + T_ATT + k * FFB_ATT_STRIDE;\n    const int n = (int)a[0];\n"
             "    for (int i = 0; i < n; ++i) ffb_linked_one(sm, (int)a[1 + i], x, y, rng, ctx, true);\n";
    s << "    (void)sm; (void)k; (void)x; (void)y; (void)rng; (void)ctx;\n}\n";
    // The final chain of normal transform k (main_template.wgsl:663-717):
    // one chain for every transform, or each its own from the table.
    s << "template <class R> __device__ __forceinline__ void ffb_finals(const float* __restrict__ sm, int k, float& x, float& y, R& rng, FfbCtx& ctx) {\n";
    if (p.fin_uniform) {
        for (int c : p.fin_chain) s << "    ffb_final_one(sm, " << c << ", x, y, rng, ctx, true);\n";
    } else {
        s << "    const float* a = sm + T_ATT + k * FFB_ATT_STRIDE + 1 + FFB_LCAP;\n    const int n = (int)a[0];\n"
             "    for (int i = 0; i < n; ++i) ffb_final_one(sm, (int)a[1 + i], x, y, rng, ctx, true);\n";
    }
    s << "    (void)sm; (void)k; (void)x; (void)y; (void)rng; (void)ctx;\n}\n";
    if (p.defer) {
        // The finals' draws by slot (FFB_FIN_SLOT0 onwards), for the
        // deferred plot: one plane of `stride` a draw.
        s << "template <class R> __device__ __forceinline__ void ffb_capture_final_draws(R& rng, float* out, unsigned long long stride) {\n";
        int m = 0;
        for (auto& fi : p.fin)
            for (size_t j = 0; j < fi.vars.size(); ++j)
                for (int d = 0; d < fi.vars[j]->draws; ++d, ++m)
                    s << "    { const float v = rng.draw(" << fi.slot[j] + d << "); out[" << m << "ull * stride] = v; }\n";
        s << "    (void)rng; (void)out; (void)stride;\n}\n";
    }
    s << kKernelsSrc << "\n";
    if (diff_window > 0) emit_diff(s, p);
    p.source = s.str();
    return p;
}

bool plan_fits(const Plan& p, const Flame& f) {
    if ((int)f.xf.size() > p.maxx) return false;
    Plan q = make_plan(f, p.rng_mode, p.math_mode, p.maxx, p.threads, p.per_xform, p.exact, p.diff_window, p.diff_ckpt, p.emit,
                       p.defer);
    return q.source == p.source;
}

std::vector<float> make_table(const Plan& p, const Flame& f) {
    std::vector<float> t((size_t)p.table_size, 0.0f);
    const int M = p.maxx;
    // utilities.wgsl:35-54: total and running sums in f32, left to right.
    float total = 0.0f;
    for (auto& x : f.xf) total += x.weight;
    t[0] = total;
    float cum = 0.0f;
    for (size_t k = 0; k < f.xf.size(); ++k) { cum += f.xf[k].weight; t[p.t_cum + k] = cum; }
    for (size_t k = f.xf.size(); k < (size_t)M; ++k) t[p.t_cum + k] = INFINITY;
    for (size_t k = 0; k < f.xf.size(); ++k) {
        const XForm& x = f.xf[k];
        const float rec[17] = {x.a, x.b, x.c, x.d, x.e, x.f, x.pa, x.pb, x.pc, x.pd, x.pe, x.pf,
                               x.post ? 1.0f : 0.0f,
                               (1.0f + x.speed) / 2.0f,                 // main_template.wgsl:499-500
                               x.color * (1.0f - x.speed) / 2.0f,
                               f.solo >= 0 && (int)k != f.solo ? 0.0f : x.opacity, x.direct_color};   // gpu/buffers.rs:531-535
        for (int fld = 0; fld < 17; ++fld) t[p.t_xf + fld * M + k] = rec[fld];
        for (size_t j = 0; j < p.normal.size(); ++j) {
            const VarDef* v = p.normal[j];
            t[p.t_vw + j * M + k] = x.var_weight(v);
            float row[kMaxVarSlots];
            x.slot_values(v, row);
            for (int q = 0; q < v->slots(); ++q) t[p.t_vp + (size_t)(p.vp_off[j] + q) * M + k] = row[q];
        }
    }
    if (p.sym_kind != 0) {
        // Post-symmetry block: copies, centre, half the pair's separation,
        // cos/sin of the axis modes' pre-rotation (-rotation), then cos/sin
        // of each point-mode copy's angle k * 2pi / order
        // (utilities.wgsl:470-568), computed here in f32.
        const PostSym& y = f.sym;
        float* q = t.data() + p.t_sym;
        q[0] = (float)y.copies();
        q[1] = y.cx; q[2] = y.cy;
        q[3] = y.distance * 0.5f;
        q[4] = std::cos(-y.rotation); q[5] = std::sin(-y.rotation);
        for (int k = 0; k < 32; ++k) {
            const float th = ((float)k * 6.28318530717958647692f) / (float)std::max(y.order, 1);
            q[6 + 2 * k] = std::cos(th);
            q[7 + 2 * k] = std::sin(th);
        }
    }
    if (p.xaos) {
        // Each previous transform's row: total, then the running sums of
        // weight_i x xaos[prev][i] in f32, left to right (utilities.wgsl:110-137).
        const size_t n = f.xf.size();
        for (int r = 0; r < M; ++r) {
            float* row = t.data() + p.t_xaos + (size_t)r * (M + 1);
            float cum = 0.0f;
            for (int i = 0; i < M; ++i) {
                if ((size_t)i < n && (size_t)r < n) { cum += f.xf[i].weight * f.xaos[(size_t)r * n + i]; row[1 + i] = cum; }
                else row[1 + i] = INFINITY;
            }
            row[0] = (size_t)r < n ? cum : 0.0f;
        }
    }
    int n_state = 0;
    const std::vector<StEntry> layout = state_layout(f, n_state);
    // Final and linked records: affine, post-affine, post flag, then the
    // weights, the parameter rows, the state bases.
    auto chain_rec = [&](const Plan::Fin& fi, const XForm& x, int kind, int pool) {
        const float rec[13] = {x.a, x.b, x.c, x.d, x.e, x.f, x.pa, x.pb, x.pc, x.pd, x.pe, x.pf, x.post ? 1.0f : 0.0f};
        for (int q = 0; q < 13; ++q) t[fi.off + q] = rec[q];
        const int nv = (int)fi.vars.size();
        for (int j = 0; j < nv; ++j) {
            t[fi.off + 13 + j] = x.var_weight(fi.vars[j]);
            float row[kMaxVarSlots];
            x.slot_values(fi.vars[j], row);
            for (int q = 0; q < fi.vars[j]->slots(); ++q) t[fi.off + 13 + nv + fi.prm_off[j] + q] = row[q];
            t[fi.off + 13 + nv + fi.prm_slots + j] = (float)state_base(layout, kind, 0, pool, fi.vars[j]);
        }
    };
    for (size_t c = 0; c < p.fin.size(); ++c) chain_rec(p.fin[c], f.fin[p.fin_pool[c]], 1, p.fin_pool[c]);
    for (size_t c = 0; c < p.lnk.size(); ++c) chain_rec(p.lnk[c], f.lnk[p.lnk_pool[c]], 3, p.lnk_pool[c]);
    // Attachments (gpu/buffers.rs:621-660) as indices into the plan's
    // linked and final lists: per normal, the linked count and entries,
    // then (chains differing) the final count and entries.
    if (p.lcap > 0 || p.fcap > 0) {
        const int stride = 2 + p.lcap + p.fcap;
        auto at = [](const std::vector<int>& pool, int c) { return (float)(std::find(pool.begin(), pool.end(), c) - pool.begin()); };
        for (size_t k = 0; k < f.xf.size(); ++k) {
            float* a = t.data() + p.t_att + k * stride;
            const XForm& x = f.xf[k];
            a[0] = (float)std::min<size_t>(x.linked_att.size(), (size_t)p.lcap);
            for (size_t i = 0; i < x.linked_att.size() && (int)i < p.lcap; ++i) a[1 + i] = at(p.lnk_pool, x.linked_att[i]);
            float* b = a + 1 + p.lcap;
            b[0] = (float)std::min<size_t>(x.final_att.size(), (size_t)p.fcap);
            for (size_t i = 0; i < x.final_att.size() && (int)i < p.fcap; ++i) b[1 + i] = at(p.fin_pool, x.final_att[i]);
        }
    }
    if (p.speed) t[p.t_speed] = f.speed_factor;
    // Each stateful normal variation's first state slot per transform.
    for (size_t j = 0; j < p.normal.size(); ++j) {
        if (p.st_row[j] < 0) continue;
        for (int k = 0; k < M; ++k)
            t[p.t_st + (size_t)p.st_row[j] * M + k] =
                (size_t)k < f.xf.size() ? (float)state_base(layout, 0, 0, k, p.normal[j]) : -1.0f;
    }
    // The state-init list, in layout order (shader_builder_v2.rs:1272-1306).
    int ni = 0;
    for (auto& e : layout) if (e.init && ni < p.n_init) t[p.t_init + ni++] = (float)e.base;
    // Subflames: total weight (at least 1e-6), whether a transform can be
    // visible, running sums in f32 (subflame.wgsl:333-361); then the inner
    // transforms' records.
    for (size_t si = 0; si < f.sub.size() && si < p.sub_blk.size(); ++si) {
        const SubFlame& S = f.sub[si];
        float* B = t.data() + p.sub_blk[si];
        float tot = 0.0f;
        bool vis = false;
        for (auto& x : S.xf) { tot += x.weight; vis = vis || (x.weight > 0.0f && x.opacity > 0.0f); }
        B[0] = std::max(tot, 1e-6f);
        B[1] = vis ? 1.0f : 0.0f;
        float cum = 0.0f;
        for (size_t i = 0; i < S.xf.size(); ++i) { cum += S.xf[i].weight; B[2 + i] = cum; }
        for (size_t tt = 0; tt < S.xf.size() + S.fin.size(); ++tt) {
            const XForm& x = inner_xf(S, tt);
            float* q = t.data() + p.sub_rec[si][tt];
            const float rec[kSubRec] = {x.a, x.b, x.c, x.d, x.e, x.f, x.pa, x.pb, x.pc, x.pd, x.pe, x.pf, x.post ? 1.0f : 0.0f,
                                        (1.0f + x.speed) * 0.5f, x.color * (1.0f - x.speed) * 0.5f, x.opacity, x.direct_color};
            for (int fld = 0; fld < kSubRec; ++fld) q[fld] = rec[fld];
            int o = kSubRec;
            for (const VarDef* v : inner_vars(f, x)) {
                q[o++] = x.var_weight(v);
                float row[kMaxVarSlots];
                x.slot_values(v, row);
                for (int r = 0; r < v->slots(); ++r) q[o++] = row[r];
                if (v->state > 0) q[o++] = (float)state_base(layout, 2, (int)si, (int)tt, v);
            }
        }
    }
    return t;
}

}  // namespace ffb
