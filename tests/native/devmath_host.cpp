// Host build of the device verify math -- TEST HARNESS ONLY.
//
// Compiles the same headers the CUDA library compiles for sm_100a
// (ultrafastsecp256k1_b200/csrc/*.cuh) with g++, so the algorithms (field /
// scalar arithmetic, safegcd, GLV, Booth windows, table build, verify logic)
// are checked against the oracle on the CPU.  The product library does not
// contain or load this file; its GPU results are checked separately by the
// -m gpu tests.
#include <stdint.h>
#include <string.h>
#include "../../ultrafastsecp256k1_b200/csrc/verify.cuh"
#include "../../ultrafastsecp256k1_b200/csrc/sign.cuh"

using namespace uf;

namespace {
struct HostTab {
    Fe x[kPTab], y[kPTab];
    void store(int k, const Fe& a, const Fe& b) { x[k] = a; y[k] = b; }
    void load(int k, Fe& a, Fe& b) const { a = x[k]; b = y[k]; }
};
struct HostGT {
    Aff pts[2 * kGTab];
    void load(int k, Fe& a, Fe& b) const { a = pts[k].x; b = pts[k].y; }
};
HostGT g_gt;
bool g_gt_ready = false;

void build_gt() {
    if (g_gt_ready) return;
    Aff G;
    gen_point(G);
    Jac acc;
    jac_set_inf(acc);
    Fe beta;
    fe_beta(beta);
    for (int i = 0; i < kGTab; ++i) {
        jac_add_aff(acc, G.x, G.y);
        jac_to_aff(g_gt.pts[i], acc);
        g_gt.pts[kGTab + i] = g_gt.pts[i];
        fe_mul(g_gt.pts[kGTab + i].x, g_gt.pts[i].x, beta);
        fe_normalize(g_gt.pts[kGTab + i].x);
    }
    g_gt_ready = true;
}

void load_words(uint32_t* w, const uint8_t* p, int n) { memcpy(w, p, 4 * n); }
}  // namespace

extern "C" {

void hm_fe_mul(const uint8_t* a, const uint8_t* b, uint8_t* out) {
    Fe x, y, r;
    be32_to_limbs(x.v, a); be32_to_limbs(y.v, b);
    fe_mul(r, x, y); fe_normalize(r); limbs_to_be32(out, r.v);
}
void hm_fe_sqr(const uint8_t* a, uint8_t* out) {
    Fe x, r;
    be32_to_limbs(x.v, a);
    fe_sqr(r, x); fe_normalize(r); limbs_to_be32(out, r.v);
}
void hm_fe_add(const uint8_t* a, const uint8_t* b, uint8_t* out) {
    Fe x, y, r;
    be32_to_limbs(x.v, a); be32_to_limbs(y.v, b);
    fe_add(r, x, y); fe_normalize(r); limbs_to_be32(out, r.v);
}
void hm_fe_sub(const uint8_t* a, const uint8_t* b, uint8_t* out) {
    Fe x, y, r;
    be32_to_limbs(x.v, a); be32_to_limbs(y.v, b);
    fe_sub(r, x, y); fe_normalize(r); limbs_to_be32(out, r.v);
}
void hm_fe_inv(const uint8_t* a, uint8_t* out) {
    Fe x, r;
    be32_to_limbs(x.v, a);
    fe_inv(r, x); fe_normalize(r); limbs_to_be32(out, r.v);
}
int hm_fe_sqrt(const uint8_t* a, uint8_t* out) {
    Fe x, r;
    be32_to_limbs(x.v, a);
    int ok = fe_sqrt(r, x);
    fe_normalize(r); limbs_to_be32(out, r.v);
    return ok;
}
void hm_sc_mul(const uint8_t* a, const uint8_t* b, uint8_t* out) {
    Sc x, y, r;
    be32_to_limbs(x.v, a); be32_to_limbs(y.v, b);
    sc_mul(r, x, y); limbs_to_be32(out, r.v);
}
void hm_sc_inv(const uint8_t* a, uint8_t* out) {
    Sc x, r;
    be32_to_limbs(x.v, a);
    sc_inv(r, x); limbs_to_be32(out, r.v);
}
// k -> k1 (16 bytes BE), k2, signs
void hm_glv(const uint8_t* k, uint8_t* k1, uint8_t* k2, uint8_t* negs) {
    Sc s;
    be32_to_limbs(s.v, k);
    GlvSplit g;
    glv_split(g, s);
    uint32_t t[8] = {0};
    for (int i = 0; i < 4; ++i) t[i] = g.k1[i];
    uint8_t buf[32];
    limbs_to_be32(buf, t); memcpy(k1, buf + 16, 16);
    for (int i = 0; i < 4; ++i) t[i] = g.k2[i];
    limbs_to_be32(buf, t); memcpy(k2, buf + 16, 16);
    negs[0] = g.neg1; negs[1] = g.neg2;
}
// booth digits of a 128-bit magnitude (16 bytes BE), w = 4 (33 digits) or the G window (UF_GWIN)
void hm_booth(const uint8_t* k16, int w, int32_t* out) {
    uint8_t buf[32] = {0};
    memcpy(buf + 16, k16, 16);
    uint32_t v[8];
    be32_to_limbs(v, buf);
    if (w == 4) { int8_t d[kNWP]; booth_recode<kWP, kNWP>(d, v); for (int i = 0; i < kNWP; ++i) out[i] = d[i]; }
    else { GDigit d[kNWG]; booth_recode<kWG, kNWG>(d, v); for (int i = 0; i < kNWG; ++i) out[i] = d[i]; }
}
// a*G + b*P for P given by x (BE) with even y; affine result or 0 for infinity
int hm_dual_mul(const uint8_t* a, const uint8_t* px32, const uint8_t* b, uint8_t* x_out, uint8_t* y_out) {
    build_gt();
    Sc sa, sb;
    be32_to_limbs(sa.v, a); be32_to_limbs(sb.v, b);
    sc_reduce_once(sa); sc_reduce_once(sb);
    Fe px, py;
    be32_to_limbs(px.v, px32);
    if (!lift_x_parity(py, px, false)) return -1;
    HostTab tab;
    Jac R;
    dual_mul(R, sa, px, py, sb, tab, g_gt);
    Aff A;
    if (!jac_to_aff(A, R)) return 0;
    limbs_to_be32(x_out, A.x.v); limbs_to_be32(y_out, A.y.v);
    return 1;
}
void hm_challenge(const uint8_t* r32, const uint8_t* p32, const uint8_t* m32, uint8_t* out) {
    uint32_t r[8], p[8], m[8], h[8];
    for (int i = 0; i < 8; ++i) {
        r[i] = ((uint32_t)r32[4*i] << 24) | ((uint32_t)r32[4*i+1] << 16) | ((uint32_t)r32[4*i+2] << 8) | r32[4*i+3];
        p[i] = ((uint32_t)p32[4*i] << 24) | ((uint32_t)p32[4*i+1] << 16) | ((uint32_t)p32[4*i+2] << 8) | p32[4*i+3];
        m[i] = ((uint32_t)m32[4*i] << 24) | ((uint32_t)m32[4*i+1] << 16) | ((uint32_t)m32[4*i+2] << 8) | m32[4*i+3];
    }
    bip340_challenge(h, r, p, m);
    for (int i = 0; i < 8; ++i) { out[4*i] = h[i] >> 24; out[4*i+1] = h[i] >> 16; out[4*i+2] = h[i] >> 8; out[4*i+3] = h[i]; }
}
void hm_ecdsa_verify_batch(const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs, size_t n, uint8_t* out) {
    build_gt();
    for (size_t i = 0; i < n; ++i) {
        uint32_t mw[8], sw[16];
        load_words(mw, msgs + 32 * i, 8);
        load_words(sw, sigs + 64 * i, 16);
        HostTab tab;
        out[i] = ecdsa_verify_one(mw, pubs + 33 * i, sw, tab, g_gt) ? 1 : 0;
    }
}
void hm_schnorr_verify_batch(const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs, size_t n, uint8_t* out) {
    build_gt();
    for (size_t i = 0; i < n; ++i) {
        uint32_t mw[8], pw[8], sw[16];
        load_words(mw, msgs + 32 * i, 8);
        load_words(pw, pubs + 32 * i, 8);
        load_words(sw, sigs + 64 * i, 16);
        HostTab tab;
        out[i] = schnorr_verify_one(mw, pw, sw, tab, g_gt) ? 1 : 0;
    }
}
}

extern "C" {
void hm_sign_batch(int kind, const uint8_t* msgs, const uint8_t* sks, const uint8_t* auxs, size_t n,
                   uint8_t* pubs, uint8_t* sigs, uint8_t* ok) {
    build_gt();
    for (size_t i = 0; i < n; ++i) {
        if (kind == 0) ok[i] = ecdsa_sign_one(pubs + 33 * i, sigs + 64 * i, msgs + 32 * i, sks + 32 * i, g_gt);
        else ok[i] = schnorr_sign_one(pubs + 32 * i, sigs + 64 * i, msgs + 32 * i, sks + 32 * i, auxs + 32 * i, g_gt);
    }
}
}
