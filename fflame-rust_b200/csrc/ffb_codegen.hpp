// ffb_codegen.hpp -- per-flame-structure CUDA source for NVRTC, and the
// float table the compiled kernel reads.
//
// The B200 counterpart of the reference's shader builder
// (src/shader_builder_v2.rs: build_definitions 1832-2030,
// build_apply_variations_2d 2525-2807, variation_call 653-681): it emits
// only the variations the flame uses, in the reference's dispatch order,
// with the NeedsRng draw of each placed at a static slot of the iteration's
// counter-based stream.  Unlike the reference's inlined-constants mode it
// bakes STRUCTURE only (which variations, in which order, how many finals);
// coefficients, weights and colours stay in a table, so flames and
// animation frames that share a structure share one compiled module.
#pragma once

#include <string>
#include <vector>

#include "ffb_flame.hpp"

namespace ffb {

enum RngMode { RNG_PCG = 0, RNG_PHILOX = 1 };
enum MathMode { MATH_PRECISE = 0, MATH_SFU = 1 };

struct Plan {
    int maxx = 0;                          // normal transforms (table capacity)
    std::vector<const VarDef*> normal;     // normal-phase variations, local order
    std::vector<int> normal_slot;          // first draw slot per normal variation (-1: none)
    std::vector<int> vp_off;               // each normal variation's first row of T_VP
    int vp_slots = 0;                      // rows of T_VP (packed parameter slots)
    struct Fin {
        std::vector<const VarDef*> vars;
        std::vector<int> slot;             // first draw slot (-1: none)
        std::vector<int> prm_off;          // parameter offset after the weights
        int prm_slots = 0;
        int off = 0;
    };
    std::vector<Fin> fin;                  // one per attached final (pool order)
    std::vector<Fin> lnk;                  // one per attached linked transform (pool order)
    std::vector<int> fin_pool, lnk_pool;   // each entry's pool index
    bool fin_uniform = true;               // every normal runs the same final chain ...
    std::vector<int> fin_chain;            // ... this one (indices into fin)
    int lcap = 0, fcap = 0;                // longest linked chain; longest final chain when they differ
    int t_att = 0;                         // per normal: linked count, lcap entries, final count, fcap entries
    int fin_slot0 = 2;                     // the finals' first draw slot
    bool has_post = false;
    int n_slots = 2;
    int table_size = 0;
    int t_cum = 0, t_xf = 0, t_vw = 0, t_vp = 0, t_fin = 0;
    int sym_kind = 0, t_sym = 0;           // post-symmetry (compile-time kind; its table block at t_sym)
    bool xaos = false;                     // xaos pick: M rows of (total, running sums) at t_xaos
    int t_xaos = 0;
    // Per-walker state of stateful variations and subflames (slots per
    // walker; rows of T_ST: each stateful normal variation's first slot per
    // transform), the state-init list (T_INIT), and whether the normal phase
    // has a variation that writes the colour register (the DC colour flow).
    int n_state = 0, n_init = 0;
    std::vector<int> st_row;               // per normal variation: its row of T_ST (-1: stateless)
    int t_st = 0, t_init = 0;
    bool dc = false;
    bool hide = false;                     // a Feature::CanHide variation anywhere in the flame
    // Speed colour mode: the walker's RGB in state slots speed_slot..+2,
    // the mix factor in the table at t_speed.
    bool speed = false;
    int speed_slot = 0, t_speed = 0;
    std::vector<int> sub_blk;              // per subflame: its block (total, any visible, running sums)
    std::vector<std::vector<int>> sub_rec; // per subflame: each inner transform's record
    int rng_mode = RNG_PHILOX;
    int math_mode = MATH_PRECISE;
    int threads = 128;
    // Emit ffb_normal_k as one straight-line case per transform.  Measured
    // slower on B200 (the inlined cases overflow the instruction cache:
    // no-instruction stalls 0.4 -> 1.7 a cycle), so off by default; the
    // union form is warp-uniform after the sorted schedule's regrouping.
    bool per_xform = false;
    bool exact = false;                    // u64 fixed-point histogram (ulonglong4 a pixel)
    bool emit = false;                     // tile-sorted accumulation: samples become records (ffb_emit)
    bool defer = false;                    // deferred plotting: the chaos kernel stores samples, ffb_plot plots them
    // Differentiable render (ffb_diff.cuh): window = iterations each sample
    // is differentiated through, ckpt = checkpoint interval; 0 = off.
    int diff_window = 0, diff_ckpt = 0;
    std::string source;                    // full NVRTC source (structure key)
};

// Structure of `f` (rng/math modes as given; maxx >= f.xf.size()).
Plan make_plan(const Flame& f, int rng_mode, int math_mode, int maxx = 0, int threads = 128, bool per_xform = false,
               bool exact = false, int diff_window = 0, int diff_ckpt = 0, bool emit = false, bool defer = false);
// The table of `f` for a plan made from a flame of the same structure.
std::vector<float> make_table(const Plan& p, const Flame& f);
// Whether `f` fits plan `p` (same structure, n_xf <= maxx).
bool plan_fits(const Plan& p, const Flame& f);

// Embedded device sources (generated into ffb_device_src.inc at build time).
extern const char* const kDeviceSrc;
extern const char* const kKernelsSrc;
extern const char* const kDiffJacSrc;
extern const char* const kDiffSrc;

}  // namespace ffb
