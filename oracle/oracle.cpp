// oracle.cpp -- CPU restatement of PrismPlan's collision-kinematics path.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h). Not linked into the product.
//
// Reference files cited below are paths inside code/gpu_planning/.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct Pair { int i, j; };

}  // namespace

struct orc_model {
    int n_dof = 0, n_joints = 0, ns = 0, na = 0;
    std::vector<double> ft, aft;          // [n_joints*16] row-major
    std::vector<float> ft32, aft32;
    std::vector<int> types, atypes, parents, id_to_dof, dfs;
    std::vector<double> sph, apx;         // [n*4]
    std::vector<float> sph32, apx32;
    std::vector<int> s2j, a2j;
    std::vector<Pair> self_pairs, apx_self_pairs;
};

struct orc_scene {
    int n_obbs = 0, n_layers = 0, max_vox = 0, esdf_mode = 0;
    std::vector<float> obb_dims, obb_pose, vparams, vpose, vfeat;
    std::vector<uint8_t> obb_en, v_en, acm, obb_acm, obb_acm_apx;
};

namespace {

// Expand {sphere_i, start, end} ranges, end inclusive
// (runtime_kinematics.cuh:258-268).
std::vector<Pair> expand_ranges(const int* r, int n) {
    std::vector<Pair> out;
    for (int k = 0; k < n; ++k)
        for (int j = r[3 * k + 1]; j <= r[3 * k + 2]; ++j) out.push_back({r[3 * k], j});
    return out;
}

// ---------------------------------------------------------------------------
// Forward kinematics (runtime_kinematics.cuh:16-89 walk; joint step formulas
// utils.cuh:571-699; FP64 form as tests/test_tree_fk_vs_cpu.py:25-58).
// T is a 3x4 affine, row-major. Joint i's world frame = frame(parent) * FT_i *
// motion(type_i, q[dof_i]); the first joint in DFS order is the identity.
// ---------------------------------------------------------------------------
template <typename F>
struct Affine { F m[12]; };

template <typename F>
inline void joint_step(const F* ft, int type, F qi, F* s) {
    // s = FT * motion(q), rows 0..2 (FT row 3 is 0 0 0 1).
    for (int k = 0; k < 12; ++k) s[k] = ft[(k / 4) * 4 + (k % 4)];
    if (type == PS_Z_ROT || type == PS_X_ROT || type == PS_Y_ROT) {
        F c = std::cos(qi), sn = std::sin(qi);
        for (int r = 0; r < 3; ++r) {
            const F* f = ft + r * 4;
            F* o = s + r * 4;
            if (type == PS_Z_ROT) {          // zrot_fn
                o[0] = f[0] * c + sn * f[1];
                o[1] = f[0] * (-sn) + c * f[1];
            } else if (type == PS_X_ROT) {   // xrot_fn
                o[1] = f[1] * c + sn * f[2];
                o[2] = f[1] * (-sn) + c * f[2];
            } else {                          // yrot_fn
                o[0] = f[0] * c + (-sn) * f[2];
                o[2] = f[0] * sn + c * f[2];
            }
        }
    } else if (type >= PS_X_PRISM && type <= PS_Z_PRISM) {   // prism_fn
        for (int r = 0; r < 3; ++r) s[r * 4 + 3] = ft[r * 4 + type] * qi + ft[r * 4 + 3];
    }
    // PS_FIXED: s = FT
}

template <typename F>
inline void compose(const F* p, const F* s, F* o) {
    // o = p * s (affine 3x4), dot4_col order (utils.cuh:709-711).
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) {
            F v = p[r * 4 + 0] * s[0 * 4 + c] + p[r * 4 + 1] * s[1 * 4 + c] + p[r * 4 + 2] * s[2 * 4 + c];
            if (c == 3) v = v + p[r * 4 + 3];
            o[r * 4 + c] = v;
        }
}

template <typename F>
void fk_frames(const orc_model& m, const F* q, bool approx, std::vector<Affine<F>>& T) {
    T.resize(m.n_joints);
    const std::vector<int>& types = approx ? m.atypes : m.types;
    for (int jj = 0; jj < m.n_joints; ++jj) {
        int i = m.dfs[jj];
        F* o = T[i].m;
        if (jj == 0) {
            for (int k = 0; k < 12; ++k) o[k] = (k % 5 == 0) ? F(1) : F(0);
            continue;
        }
        F ft[16];
        if (sizeof(F) == sizeof(double)) {
            const std::vector<double>& src = approx ? m.aft : m.ft;
            for (int k = 0; k < 16; ++k) ft[k] = (F)src[i * 16 + k];
        } else {
            const std::vector<float>& src = approx ? m.aft32 : m.ft32;
            for (int k = 0; k < 16; ++k) ft[k] = (F)src[i * 16 + k];
        }
        int dof = m.id_to_dof[i];
        F qi = dof >= 0 ? q[dof] : F(0);
        F s[12];
        joint_step<F>(ft, types[i], qi, s);
        compose<F>(T[m.parents[i]].m, s, o);
    }
}

template <typename F>
inline void sphere_world(const Affine<F>& T, F x, F y, F z, F* p) {
    // runtime_kinematics.cuh:79-83
    for (int r = 0; r < 3; ++r)
        p[r] = T.m[r * 4 + 0] * x + T.m[r * 4 + 1] * y + T.m[r * 4 + 2] * z + T.m[r * 4 + 3];
}

// ---------------------------------------------------------------------------
// Scene primitives (scene_collision.cuh)
// ---------------------------------------------------------------------------
template <typename F>
inline void to_local(const float* pose, F sx, F sy, F sz, F& lx, F& ly, F& lz) {
    // transform_sphere_to_local, scene_collision.cuh:24-51
    F qw = pose[3], qx = pose[4], qy = pose[5], qz = pose[6];
    F tx = F(2) * (qy * sz - qz * sy);
    F ty = F(2) * (qz * sx - qx * sz);
    F tz = F(2) * (qx * sy - qy * sx);
    F rx = sx + qw * tx + (qy * tz - qz * ty);
    F ry = sy + qw * ty + (qz * tx - qx * tz);
    F rz = sz + qw * tz + (qx * ty - qy * tx);
    lx = rx + (F)pose[0];
    ly = ry + (F)pose[1];
    lz = rz + (F)pose[2];
}

// Box outside-distance squared and SDF in the OBB frame.
template <typename F>
inline void box_terms(const float* dims, F lx, F ly, F lz, F& dist_sq, F& sdf) {
    F hx = (F)dims[0] * F(0.5), hy = (F)dims[1] * F(0.5), hz = (F)dims[2] * F(0.5);
    F qx = std::fabs(lx) - hx, qy = std::fabs(ly) - hy, qz = std::fabs(lz) - hz;
    F ox = std::max(qx, F(0)), oy = std::max(qy, F(0)), oz = std::max(qz, F(0));
    dist_sq = ox * ox + oy * oy + oz * oz;                    // scene_collision.cuh:72-76
    F inside = std::min(std::max(qx, std::max(qy, qz)), F(0));  // :100-111
    sdf = std::sqrt(dist_sq) + inside;
}

template <typename F>
inline bool obb_any(const orc_scene& s, const F* p, F sr, int sphere_idx, const uint8_t* acm,
                    double* gap) {
    // sphere_obb_in_collision (scene_collision.cuh:118-138); gap tracks
    // min(|c| - sr) for the FP64 distance to contact.
    bool hit = false;
    for (int o = 0; o < s.n_obbs; ++o) {
        if (s.obb_en[o] == 0) continue;
        if (sphere_idx >= 0 && acm && acm[(size_t)sphere_idx * s.n_obbs + o] == 0) continue;
        F lx, ly, lz, dsq, sdf;
        to_local<F>(&s.obb_pose[o * 8], p[0], p[1], p[2], lx, ly, lz);
        box_terms<F>(&s.obb_dims[o * 4], lx, ly, lz, dsq, sdf);
        if (dsq < sr * sr) hit = true;
        if (gap) *gap = std::min(*gap, (double)std::sqrt(dsq) - (double)sr);
        if (hit && !gap) return true;
    }
    return hit;
}

template <typename F>
inline F obb_clearance(const orc_scene& s, const F* p, F sr, int sphere_idx, const uint8_t* acm) {
    // sphere_obb_clearance (scene_collision.cuh:148-167)
    F best = F(1000);
    for (int o = 0; o < s.n_obbs; ++o) {
        if (s.obb_en[o] == 0) continue;
        if (sphere_idx >= 0 && acm && acm[(size_t)sphere_idx * s.n_obbs + o] == 0) continue;
        F lx, ly, lz, dsq, sdf;
        to_local<F>(&s.obb_pose[o * 8], p[0], p[1], p[2], lx, ly, lz);
        box_terms<F>(&s.obb_dims[o * 4], lx, ly, lz, dsq, sdf);
        best = std::min(best, sdf - sr);
    }
    return best;
}

inline int robust_floor(float x) {
    // robust_floor_scalar (scene_collision.cuh:192-200)
    float nearest = std::round(x);
    float diff = x - nearest;
    if (diff >= 1e-4f) return (int)std::floor(x);
    return (int)std::nearbyint(nearest);
}

// One ESDF layer lookup. Returns false if the sphere is out of range /
// unobserved for this layer; otherwise distance ("positive = inside").
// Nearest mode restates scene_collision.cuh:215-256 (index math in FP32 as the
// reference). Trilinear mode interpolates the 8 voxels around the continuous
// index with the same guard and skips if any corner is unobserved.
template <typename F>
inline bool esdf_lookup(const orc_scene& s, int layer, const F* p, F& distance) {
    const float* prm = &s.vparams[layer * 4];
    const float* pose = &s.vpose[layer * 8];
    float gdx = prm[0], gdy = prm[1], gdz = prm[2], vs = prm[3];
    if (vs <= 0.0f) return false;
    F lx, ly, lz;
    to_local<F>(pose, p[0], p[1], p[2], lx, ly, lz);
    float inv_vs = 1.0f / vs;
    int nx = robust_floor(gdx * inv_vs) + 1, ny = robust_floor(gdy * inv_vs) + 1,
        nz = robust_floor(gdz * inv_vs) + 1;
    const float* feat = &s.vfeat[(size_t)layer * s.max_vox];
    const int B = 2;
    if (s.esdf_mode == PS_ESDF_NEAREST) {
        int ix = (int)(((float)lx + gdx * 0.5f) * inv_vs);
        int iy = (int)(((float)ly + gdy * 0.5f) * inv_vs);
        int iz = (int)(((float)lz + gdz * 0.5f) * inv_vs);
        if (ix >= nx - B || iy >= ny - B || iz >= nz - B || ix <= B || iy <= B || iz <= B) return false;
        long long li = (long long)ix * ny * nz + (long long)iy * nz + iz;
        if (li >= s.max_vox) return false;
        float d = feat[li];
        if (d <= -1000.0f + 1.0f) return false;
        distance = (F)d;
        return true;
    }
    F gx = (lx + (F)gdx * F(0.5)) * (F)inv_vs, gy = (ly + (F)gdy * F(0.5)) * (F)inv_vs,
      gz = (lz + (F)gdz * F(0.5)) * (F)inv_vs;
    F fx0 = std::floor(gx), fy0 = std::floor(gy), fz0 = std::floor(gz);
    if (!(fx0 > F(B) && fy0 > F(B) && fz0 > F(B) && fx0 + 1 < F(nx - B) && fy0 + 1 < F(ny - B) &&
          fz0 + 1 < F(nz - B)))
        return false;
    int ix = (int)fx0, iy = (int)fy0, iz = (int)fz0;
    F fx = gx - fx0, fy = gy - fy0, fz = gz - fz0;
    F v[8];
    for (int c = 0; c < 8; ++c) {
        long long li = (long long)(ix + (c & 1)) * ny * nz + (long long)(iy + ((c >> 1) & 1)) * nz +
                       (iz + ((c >> 2) & 1));
        if (li >= s.max_vox) return false;
        float d = feat[li];
        if (d <= -1000.0f + 1.0f) return false;
        v[c] = (F)d;
    }
    F x00 = v[0] + fx * (v[1] - v[0]), x10 = v[2] + fx * (v[3] - v[2]);
    F x01 = v[4] + fx * (v[5] - v[4]), x11 = v[6] + fx * (v[7] - v[6]);
    F y0 = x00 + fy * (x10 - x00), y1 = x01 + fy * (x11 - x01);
    distance = y0 + fz * (y1 - y0);
    return true;
}

template <typename F>
inline bool esdf_any(const orc_scene& s, const F* p, F sr, int sphere_idx) {
    // sphere_esdf_in_collision (scene_collision.cuh:202-266)
    for (int l = 0; l < s.n_layers; ++l) {
        if (s.v_en[l] == 0) continue;
        if (sphere_idx >= 0 && !s.acm.empty() && s.acm[(size_t)sphere_idx * s.n_layers + l] == 0)
            continue;
        F d;
        if (!esdf_lookup<F>(s, l, p, d)) continue;
        if (d > -sr) return true;
    }
    return false;
}

template <typename F>
inline F esdf_clearance(const orc_scene& s, const F* p, F sr, int sphere_idx) {
    // sphere_esdf_clearance (scene_collision.cuh:276-331)
    F best = F(1000);
    for (int l = 0; l < s.n_layers; ++l) {
        if (s.v_en[l] == 0) continue;
        if (sphere_idx >= 0 && !s.acm.empty() && s.acm[(size_t)sphere_idx * s.n_layers + l] == 0)
            continue;
        F d;
        if (!esdf_lookup<F>(s, l, p, d)) continue;
        best = std::min(best, -d - sr);
    }
    return best;
}

// ---------------------------------------------------------------------------
// Two-phase verdict (two_phase_cc.cuh:57-138) for one configuration.
// ---------------------------------------------------------------------------
template <typename F>
struct ConfigResult {
    bool hit = false;
    double clearance = 1000.0;
    double gap = 1e30;
};

template <typename F>
void eval_config(const orc_model& m, const orc_scene& s, const float* qf, F margin, unsigned flags,
                 ConfigResult<F>& res, bool want_gap) {
    F q[PS_MAX_DOF];
    for (int d = 0; d < m.n_dof; ++d) q[d] = (F)qf[d];
    std::vector<Affine<F>> T, TA;
    fk_frames<F>(m, q, false, T);
    fk_frames<F>(m, q, true, TA);
    const uint8_t* acm_apx = s.obb_acm_apx.empty() ? nullptr : s.obb_acm_apx.data();
    const uint8_t* acm = s.obb_acm.empty() ? nullptr : s.obb_acm.data();

    // approximate pass: flags per joint (scene_collision.cuh:584-631)
    std::vector<char> jic(m.n_joints, 0);
    bool gate_off = (flags & PS_NO_GATE) != 0;
    std::vector<F> apos(m.na * 3);
    for (int a = 0; a < m.na; ++a) {
        F x = (F)m.apx[a * 4], y = (F)m.apx[a * 4 + 1], z = (F)m.apx[a * 4 + 2];
        F r = (F)m.apx[a * 4 + 3];
        if (sizeof(F) == 4) { x = m.apx32[a * 4]; y = m.apx32[a * 4 + 1]; z = m.apx32[a * 4 + 2]; r = m.apx32[a * 4 + 3]; }
        F p[3];
        sphere_world<F>(TA[m.a2j[a]], x, y, z, p);
        apos[a * 3] = p[0]; apos[a * 3 + 1] = p[1]; apos[a * 3 + 2] = p[2];
        F sr = r + margin;
        if (!gate_off && (obb_any<F>(s, p, sr, -1, acm_apx, nullptr) || esdf_any<F>(s, p, sr, -1)))
            jic[m.a2j[a]] = 1;
    }
    // exact pass, gated per joint (scene_collision.cuh:519-567)
    std::vector<F> pos(m.ns * 3);
    bool hit = false;
    double gap = 1e30;
    double clr = 1000.0;
    for (int i = 0; i < m.ns; ++i) {
        F x = (F)m.sph[i * 4], y = (F)m.sph[i * 4 + 1], z = (F)m.sph[i * 4 + 2], r = (F)m.sph[i * 4 + 3];
        if (sizeof(F) == 4) { x = m.sph32[i * 4]; y = m.sph32[i * 4 + 1]; z = m.sph32[i * 4 + 2]; r = m.sph32[i * 4 + 3]; }
        F p[3];
        sphere_world<F>(T[m.s2j[i]], x, y, z, p);
        pos[i * 3] = p[0]; pos[i * 3 + 1] = p[1]; pos[i * 3 + 2] = p[2];
        F sr = r + margin;
        if (gate_off || jic[m.s2j[i]]) {
            double g = 1e30;
            bool h = obb_any<F>(s, p, sr, i, acm, want_gap ? &g : nullptr) || esdf_any<F>(s, p, sr, i);
            hit = hit || h;
            gap = std::min(gap, g);
        }
        if (flags & PS_CLEARANCE_OBB) clr = std::min(clr, (double)obb_clearance<F>(s, p, sr, i, acm));
        if (flags & PS_CLEARANCE_ESDF) clr = std::min(clr, (double)esdf_clearance<F>(s, p, sr, i));
    }
    // self (runtime_kinematics.cuh:248-284, 382-416; two_phase_cc.cuh:109-130).
    // With want_gap every pair is visited and gap also takes the distance to
    // contact |d - (r_i + r_j)| of each approximate and exact pair, so that a
    // self verdict flip can be reported with its distance to contact.
    if ((flags & PS_CHECK_SELF) && !hit) {
        bool need = gate_off;
        for (const Pair& pr : m.apx_self_pairs) {
            if (need && !want_gap) break;
            F dx = apos[pr.i * 3] - apos[pr.j * 3], dy = apos[pr.i * 3 + 1] - apos[pr.j * 3 + 1],
              dz = apos[pr.i * 3 + 2] - apos[pr.j * 3 + 2];
            F rs = (F)m.apx[pr.i * 4 + 3] + (F)m.apx[pr.j * 4 + 3];
            if (sizeof(F) == 4) rs = m.apx32[pr.i * 4 + 3] + m.apx32[pr.j * 4 + 3];
            if (dx * dx + dy * dy + dz * dz - rs * rs < F(0)) need = true;
            if (want_gap) gap = std::min(gap, std::fabs(std::sqrt((double)(dx * dx + dy * dy + dz * dz)) - (double)rs));
        }
        if (need || want_gap) {
            bool self_hit = false;
            for (const Pair& pr : m.self_pairs) {
                F dx = pos[pr.i * 3] - pos[pr.j * 3], dy = pos[pr.i * 3 + 1] - pos[pr.j * 3 + 1],
                  dz = pos[pr.i * 3 + 2] - pos[pr.j * 3 + 2];
                F rs = (F)m.sph[pr.i * 4 + 3] + (F)m.sph[pr.j * 4 + 3];
                if (sizeof(F) == 4) rs = m.sph32[pr.i * 4 + 3] + m.sph32[pr.j * 4 + 3];
                F sum = dx * dx + dy * dy + dz * dz;
                if (want_gap) gap = std::min(gap, std::fabs(std::sqrt((double)sum) - (double)rs));
                if (sum - rs * rs < F(0)) {
                    self_hit = true;
                    if (!want_gap) break;
                }
            }
            hit = need && self_hit;
        }
    }
    res.hit = hit;
    res.gap = gap;
    res.clearance = clr;
}

template <typename Fn>
void parallel_for(int n, int threads, Fn fn) {
    if (threads <= 1 || n < 2) {
        for (int i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    const int chunk = std::max(1, n / (threads * 16));
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&]() {
            for (;;) {
                int b = next.fetch_add(chunk);
                if (b >= n) break;
                int e = std::min(n, b + chunk);
                for (int i = b; i < e; ++i) fn(i);
            }
        });
    for (auto& th : pool) th.join();
}

// Per-waypoint state cost (chomp.cu:151-188) at precision F.
template <typename F>
F state_cost(const orc_model& m, const orc_scene& s, const F* q, F w, F wm, F sm, int include_self) {
    std::vector<Affine<F>> T;
    fk_frames<F>(m, q, false, T);
    const uint8_t* acm = s.obb_acm.empty() ? nullptr : s.obb_acm.data();
    std::vector<F> pos(m.ns * 3);
    F esdf_sum = 0, obb_sum = 0;
    for (int i = 0; i < m.ns; ++i) {
        F x = (F)m.sph[i * 4], y = (F)m.sph[i * 4 + 1], z = (F)m.sph[i * 4 + 2], r = (F)m.sph[i * 4 + 3];
        if (sizeof(F) == 4) { x = m.sph32[i * 4]; y = m.sph32[i * 4 + 1]; z = m.sph32[i * 4 + 2]; r = m.sph32[i * 4 + 3]; }
        F p[3];
        sphere_world<F>(T[m.s2j[i]], x, y, z, p);
        pos[i * 3] = p[0]; pos[i * 3 + 1] = p[1]; pos[i * 3 + 2] = p[2];
        esdf_sum += std::max(F(0), wm - esdf_clearance<F>(s, p, r, i));   // scene_collision.cuh:394-438
        obb_sum += std::max(F(0), wm - obb_clearance<F>(s, p, r, i, acm)); // :449-495
    }
    F self = 0;
    if (include_self) {   // self_min_hinge_runtime, runtime_kinematics.cuh:294-329
        F mn = F(1000);
        for (const Pair& pr : m.self_pairs) {
            F dx = pos[pr.i * 3] - pos[pr.j * 3], dy = pos[pr.i * 3 + 1] - pos[pr.j * 3 + 1],
              dz = pos[pr.i * 3 + 2] - pos[pr.j * 3 + 2];
            F ri = (F)m.sph[pr.i * 4 + 3], rj = (F)m.sph[pr.j * 4 + 3];
            if (sizeof(F) == 4) { ri = m.sph32[pr.i * 4 + 3]; rj = m.sph32[pr.j * 4 + 3]; }
            F clr = std::sqrt(dx * dx + dy * dy + dz * dz) - (ri + rj);
            mn = std::min(mn, clr);
        }
        self = std::max(F(0), sm - mn);
    }
    return w * (esdf_sum + obb_sum + self);
}

}  // namespace

extern "C" {

orc_model* orc_model_create(const ps_model_desc* d) {
    if (!d || d->n_joints <= 0 || d->n_joints > PS_MAX_JOINTS || d->n_dof <= 0 || d->n_dof > PS_MAX_DOF)
        return nullptr;
    orc_model* m = new orc_model();
    m->n_dof = d->n_dof;
    m->n_joints = d->n_joints;
    m->ns = d->n_spheres;
    m->na = d->n_approx_spheres;
    int nj = d->n_joints;
    m->ft.assign(d->fixed_transforms, d->fixed_transforms + nj * 16);
    m->ft32.assign(d->fixed_transforms, d->fixed_transforms + nj * 16);
    const float* aft = d->approx_fixed_transforms ? d->approx_fixed_transforms : d->fixed_transforms;
    m->aft.assign(aft, aft + nj * 16);
    m->aft32.assign(aft, aft + nj * 16);
    m->types.assign(d->joint_types, d->joint_types + nj);
    const int* at = d->approx_joint_types ? d->approx_joint_types : d->joint_types;
    m->atypes.assign(at, at + nj);
    // serial defaults (robot_model.cuh:204-236)
    m->parents.resize(nj); m->id_to_dof.resize(nj); m->dfs.resize(nj);
    for (int i = 0; i < nj; ++i) {
        m->parents[i] = d->joint_parents ? d->joint_parents[i] : (i > 0 ? i - 1 : 0);
        m->id_to_dof[i] = d->joint_id_to_dof ? d->joint_id_to_dof[i] : i - 1;
        m->dfs[i] = d->dfs_order ? d->dfs_order[i] : i;
    }
    m->sph.assign(d->spheres, d->spheres + m->ns * 4);
    m->sph32.assign(d->spheres, d->spheres + m->ns * 4);
    m->s2j.assign(d->sphere_to_joint, d->sphere_to_joint + m->ns);
    if (m->na > 0) {
        m->apx.assign(d->approx_spheres, d->approx_spheres + m->na * 4);
        m->apx32.assign(d->approx_spheres, d->approx_spheres + m->na * 4);
        m->a2j.assign(d->approx_sphere_to_joint, d->approx_sphere_to_joint + m->na);
    }
    if (d->n_self_cc_ranges > 0) m->self_pairs = expand_ranges(d->self_cc_ranges, d->n_self_cc_ranges);
    if (d->n_approx_self_cc_ranges > 0)
        m->apx_self_pairs = expand_ranges(d->approx_self_cc_ranges, d->n_approx_self_cc_ranges);
    return m;
}

void orc_model_destroy(orc_model* m) { delete m; }

orc_scene* orc_scene_create(const float* obb_dims, const float* obb_pose, const uint8_t* obb_enable,
                            int n_obbs, const float* voxel_params, const float* voxel_pose,
                            const uint8_t* voxel_enable, const float* voxel_features, int n_layers,
                            int max_vox, const uint8_t* acm, const uint8_t* obb_acm,
                            const uint8_t* obb_acm_apx, int esdf_mode) {
    orc_scene* s = new orc_scene();
    s->n_obbs = n_obbs;
    s->n_layers = n_layers;
    s->max_vox = max_vox;
    s->esdf_mode = esdf_mode;
    if (n_obbs > 0) {
        s->obb_dims.assign(obb_dims, obb_dims + n_obbs * 4);
        s->obb_pose.assign(obb_pose, obb_pose + n_obbs * 8);
        if (obb_enable) s->obb_en.assign(obb_enable, obb_enable + n_obbs);
        else s->obb_en.assign(n_obbs, 1);
    }
    if (n_layers > 0) {
        s->vparams.assign(voxel_params, voxel_params + n_layers * 4);
        s->vpose.assign(voxel_pose, voxel_pose + n_layers * 8);
        if (voxel_enable) s->v_en.assign(voxel_enable, voxel_enable + n_layers);
        else s->v_en.assign(n_layers, 1);
        s->vfeat.assign(voxel_features, voxel_features + (size_t)n_layers * max_vox);
    }
    // The masks' sizes depend on the model; orc_scene_set_masks copies them.
    (void)acm; (void)obb_acm; (void)obb_acm_apx;
    return s;
}

void orc_scene_destroy(orc_scene* s) { delete s; }

}  // extern "C"

// Masks need the model's sphere counts; the Python side passes them through
// this helper after orc_scene_create.
extern "C" void orc_scene_set_masks(orc_scene* s, const uint8_t* acm, int n_acm,
                                    const uint8_t* obb_acm, int n_obb_acm,
                                    const uint8_t* obb_acm_apx, int n_obb_acm_apx) {
    // each call replaces all three masks; NULL (or empty) means none
    s->acm.clear();
    s->obb_acm.clear();
    s->obb_acm_apx.clear();
    if (acm && n_acm > 0) s->acm.assign(acm, acm + n_acm);
    if (obb_acm && n_obb_acm > 0) s->obb_acm.assign(obb_acm, obb_acm + n_obb_acm);
    if (obb_acm_apx && n_obb_acm_apx > 0) s->obb_acm_apx.assign(obb_acm_apx, obb_acm_apx + n_obb_acm_apx);
}

extern "C" void orc_fk_spheres(const orc_model* m, const float* q, int n, int prec, double* out) {
    for (int c = 0; c < n; ++c) {
        if (prec == 64) {
            double qd[PS_MAX_DOF];
            for (int d = 0; d < m->n_dof; ++d) qd[d] = q[c * m->n_dof + d];
            std::vector<Affine<double>> T;
            fk_frames<double>(*m, qd, false, T);
            for (int i = 0; i < m->ns; ++i) {
                double p[3];
                sphere_world<double>(T[m->s2j[i]], m->sph[i * 4], m->sph[i * 4 + 1], m->sph[i * 4 + 2], p);
                for (int k = 0; k < 3; ++k) out[((size_t)c * m->ns + i) * 3 + k] = p[k];
            }
        } else {
            std::vector<Affine<float>> T;
            fk_frames<float>(*m, q + c * m->n_dof, false, T);
            for (int i = 0; i < m->ns; ++i) {
                float p[3];
                sphere_world<float>(T[m->s2j[i]], m->sph32[i * 4], m->sph32[i * 4 + 1], m->sph32[i * 4 + 2], p);
                for (int k = 0; k < 3; ++k) out[((size_t)c * m->ns + i) * 3 + k] = p[k];
            }
        }
    }
}

extern "C" int orc_check_configs(const orc_model* m, const orc_scene* s, const float* q, int n,
                                 float margin, unsigned flags, int prec, int threads, uint8_t* hit,
                                 double* clearance, double* gap) {
    parallel_for(n, threads, [&](int c) {
        if (prec == 64) {
            ConfigResult<double> r;
            eval_config<double>(*m, *s, q + (size_t)c * m->n_dof, (double)margin, flags, r, gap != nullptr);
            hit[c] = r.hit;
            if (clearance) clearance[c] = r.clearance;
            if (gap) gap[c] = r.gap;
        } else {
            ConfigResult<float> r;
            eval_config<float>(*m, *s, q + (size_t)c * m->n_dof, margin, flags, r, gap != nullptr);
            hit[c] = r.hit;
            if (clearance) clearance[c] = r.clearance;
            if (gap) gap[c] = r.gap;
        }
    });
    return 0;
}

extern "C" int orc_check_edges(const orc_model* m, const orc_scene* s, const float* from,
                               const float* to, const int* G, int n_edges, float margin,
                               int check_self, int compute_clearance, int early_exit, int prec,
                               int threads, uint8_t* valid, double* cost, double* clearance,
                               double* gap, long long* samples_done) {
    std::atomic<long long> done{0};
    unsigned flags = (check_self ? PS_CHECK_SELF : 0u) | (compute_clearance ? PS_CLEARANCE_ESDF : 0u);
    parallel_for(n_edges, threads, [&](int e) {
        const int D = m->n_dof;
        const float* a = from + (size_t)e * D;
        const float* b = to + (size_t)e * D;
        // L2 length in FP32 (edge_eval.cuh:104-106)
        float len2 = 0.0f;
        for (int i = 0; i < D; ++i) { float d = b[i] - a[i]; len2 = std::fma(d, d, len2); }
        float len = std::sqrt(len2);
        int g = G[e];
        bool bad = false;
        double egap = 1e30, eclr = (double)FLT_MAX;
        long long cnt = 0;
        // Samples j = 1..G (t = j/G); slots past G in the last block of 16 take
        // t = 0, the start configuration, and their verdict counts
        // (edge_eval.cuh:110-130): it is evaluated last, as j = G + 1.
        const int extra = (g > 0 && g % 16 != 0) ? 1 : 0;
        for (int j = 1; j <= g + extra; ++j) {
            float t = (j <= g) ? (float)j / (float)g : 0.0f;
            float qs[PS_MAX_DOF];
            for (int i = 0; i < D; ++i) qs[i] = std::fma(t, b[i] - a[i], a[i]);
            ++cnt;
            bool h;
            double cl, gp;
            if (prec == 64) {
                ConfigResult<double> r;
                eval_config<double>(*m, *s, qs, (double)margin, flags, r, gap != nullptr);
                h = r.hit; cl = r.clearance; gp = r.gap;
            } else {
                ConfigResult<float> r;
                eval_config<float>(*m, *s, qs, margin, flags, r, gap != nullptr);
                h = r.hit; cl = r.clearance; gp = r.gap;
            }
            egap = std::min(egap, gp);
            if (compute_clearance && j <= g) eclr = std::min(eclr, cl);
            if (h) {
                bad = true;
                if (early_exit) break;
            }
        }
        done += cnt;
        valid[e] = bad ? 0 : 1;
        cost[e] = bad ? (double)FLT_MAX : (double)len;
        if (clearance) clearance[e] = compute_clearance ? eclr : (double)FLT_MAX;
        if (gap) gap[e] = egap;
    });
    if (samples_done) *samples_done = done.load();
    return 0;
}

extern "C" int orc_state_cost(const orc_model* m, const orc_scene* s, const float* q, int n, float w,
                              float wm, float sm, int include_self, int prec, int threads,
                              double* out) {
    parallel_for(n, threads, [&](int c) {
        const float* qc = q + (size_t)c * m->n_dof;
        if (prec == 64) {
            double qd[PS_MAX_DOF];
            for (int d = 0; d < m->n_dof; ++d) qd[d] = qc[d];
            out[c] = state_cost<double>(*m, *s, qd, w, wm, sm, include_self);
        } else {
            out[c] = state_cost<float>(*m, *s, qc, w, wm, sm, include_self);
        }
    });
    return 0;
}

extern "C" double orc_state_cost_d(const orc_model* m, const orc_scene* s, const double* q, double w,
                                   double wm, double sm, int include_self) {
    return state_cost<double>(*m, *s, q, w, wm, sm, include_self);
}

// Distance (metres) from p to the nearest face of layer l's voxel lattice:
// where the nearest lookup's voxel, or the trilinear lookup's cell, changes
// (the guard band's edges lie on the same lattice).
static double esdf_face_distance(const orc_scene& s, int layer, const double* p) {
    const float* prm = &s.vparams[layer * 4];
    const double vs = prm[3];
    if (vs <= 0.0) return 1e30;
    double l[3];
    to_local<double>(&s.vpose[layer * 8], p[0], p[1], p[2], l[0], l[1], l[2]);
    double best = 1e30;
    for (int k = 0; k < 3; ++k) {
        const double g = (l[k] + prm[k] * 0.5) / vs;
        const double f = g - std::floor(g);
        best = std::min(best, std::min(f, 1.0 - f) * vs);
    }
    return best;
}

extern "C" double orc_state_cost_kink_distance(const orc_model* m, const orc_scene* s, const double* q,
                                               double wm, double sm, int include_self) {
    std::vector<Affine<double>> T;
    fk_frames<double>(*m, q, false, T);
    const uint8_t* acm = s->obb_acm.empty() ? nullptr : s->obb_acm.data();
    double kd = 1e30;
    std::vector<double> pos(m->ns * 3);
    for (int i = 0; i < m->ns; ++i) {
        double p[3];
        sphere_world<double>(T[m->s2j[i]], m->sph[i * 4], m->sph[i * 4 + 1], m->sph[i * 4 + 2], p);
        pos[i * 3] = p[0]; pos[i * 3 + 1] = p[1]; pos[i * 3 + 2] = p[2];
        double r = m->sph[i * 4 + 3];
        double best = 1000.0, second = 1000.0;
        int best_o = -1;
        double best_q[3] = {0, 0, 0}, best_l[3] = {0, 0, 0};
        for (int o = 0; o < s->n_obbs; ++o) {
            if (s->obb_en[o] == 0) continue;
            if (acm && acm[(size_t)i * s->n_obbs + o] == 0) continue;
            double l[3], dsq, sdf;
            to_local<double>(&s->obb_pose[o * 8], p[0], p[1], p[2], l[0], l[1], l[2]);
            box_terms<double>(&s->obb_dims[o * 4], l[0], l[1], l[2], dsq, sdf);
            double c = sdf - r;
            if (c < best) {
                second = best; best = c; best_o = o;
                for (int k = 0; k < 3; ++k) {
                    best_l[k] = l[k];
                    best_q[k] = std::fabs(l[k]) - s->obb_dims[o * 4 + k] * 0.5;
                }
            } else if (c < second) {
                second = c;
            }
        }
        // ESDF: hinge activation of the min over layers, ties between layers,
        // and the voxel faces of the minimising layer
        if (s->n_layers > 0) {
            double eb = 1000.0, e2 = 1000.0;
            int el = -1;
            for (int l = 0; l < s->n_layers; ++l) {
                if (s->v_en[l] == 0) continue;
                if (!s->acm.empty() && s->acm[(size_t)i * s->n_layers + l] == 0) continue;
                double d;
                if (!esdf_lookup<double>(*s, l, p, d)) continue;
                const double c = -d - r;
                if (c < eb) { e2 = eb; eb = c; el = l; } else if (c < e2) { e2 = c; }
            }
            if (el >= 0) {
                kd = std::min(kd, std::fabs(wm - eb));
                if (eb < wm) {   // active: the value (nearest) or the gradient (trilinear) jumps across faces
                    kd = std::min(kd, e2 - eb);
                    kd = std::min(kd, esdf_face_distance(*s, el, p));
                }
            }
        }
        if (best_o < 0) continue;
        kd = std::min(kd, std::fabs(wm - best));       // hinge activation
        if (best < wm) {                                // active: min tie + box regions
            kd = std::min(kd, second - best);
            bool inside = best_q[0] < 0 && best_q[1] < 0 && best_q[2] < 0;
            for (int k = 0; k < 3; ++k) {
                kd = std::min(kd, std::fabs(best_q[k]));
                kd = std::min(kd, std::fabs(best_l[k]));
            }
            if (inside) {
                kd = std::min(kd, std::fabs(best_q[0] - best_q[1]));
                kd = std::min(kd, std::fabs(best_q[1] - best_q[2]));
                kd = std::min(kd, std::fabs(best_q[0] - best_q[2]));
            }
        }
    }
    if (include_self && !m->self_pairs.empty()) {
        double b1 = 1000.0, b2 = 1000.0;
        for (const Pair& pr : m->self_pairs) {
            double dx = pos[pr.i * 3] - pos[pr.j * 3], dy = pos[pr.i * 3 + 1] - pos[pr.j * 3 + 1],
                   dz = pos[pr.i * 3 + 2] - pos[pr.j * 3 + 2];
            double c = std::sqrt(dx * dx + dy * dy + dz * dz) - (m->sph[pr.i * 4 + 3] + m->sph[pr.j * 4 + 3]);
            if (c < b1) { b2 = b1; b1 = c; } else if (c < b2) { b2 = c; }
        }
        kd = std::min(kd, std::fabs(sm - b1));
        if (b1 < sm) kd = std::min(kd, b2 - b1);
    }
    return kd;
}

extern "C" int orc_state_cost_fd_grad(const orc_model* m, const orc_scene* s, const float* q, int n,
                                      float w, float wm, float sm, int include_self, double h,
                                      int threads, double* grad) {
    const int D = m->n_dof;
    parallel_for(n, threads, [&](int c) {
        double qd[PS_MAX_DOF];
        for (int d = 0; d < D; ++d) qd[d] = q[(size_t)c * D + d];
        for (int d = 0; d < D; ++d) {
            double save = qd[d];
            qd[d] = save + h;
            double cp = state_cost<double>(*m, *s, qd, w, wm, sm, include_self);
            qd[d] = save - h;
            double cm = state_cost<double>(*m, *s, qd, w, wm, sm, include_self);
            qd[d] = save;
            grad[(size_t)c * D + d] = (cp - cm) / (2.0 * h);
        }
    });
    return 0;
}

extern "C" void orc_control_cost_R(int T, double dt, double* R) {
    // chomp_precompute.cpp:20-37: A is the 5-point acceleration stencil
    // {-1,16,-30,16,-1}/12 / dt^2 on a grid padded by 6 each side;
    // R = dt * A^T A, central T x T block.
    const int pad = 6, Np = T + 2 * pad;
    const double coeff[7] = {0.0, -1.0 / 12, 16.0 / 12, -30.0 / 12, 16.0 / 12, -1.0 / 12, 0.0};
    const double inv_dt2 = 1.0 / (dt * dt);
    std::vector<double> A((size_t)Np * Np, 0.0);
    for (int i = 0; i < Np; ++i)
        for (int j = -3; j <= 3; ++j) {
            int idx = i + j;
            if (idx < 0 || idx >= Np) continue;
            A[(size_t)i * Np + idx] = inv_dt2 * coeff[j + 3];
        }
    for (int a = 0; a < T; ++a)
        for (int b = 0; b < T; ++b) {
            double acc = 0.0;
            int ia = a + pad, ib = b + pad;
            for (int k = 0; k < Np; ++k) acc += A[(size_t)k * Np + ia] * A[(size_t)k * Np + ib];
            R[(size_t)a * T + b] = dt * acc;
        }
}
