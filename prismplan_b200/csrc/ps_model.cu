// ps_model.cu -- robot model upload, scene validation, error plumbing and the
// shared-memory staging routines.
//
// Host side of ppln::RobotModelDevice::create / destroy
// (code/gpu_planning/cpp/src/planning/robot_model.cuh:91-293), re-laid out for
// the B200 kernels: the whole model is ONE device allocation whose "core"
// (header, per-joint records in DFS visit order, sphere tables re-ordered by
// joint) is copied into shared memory by a single bulk async copy per block.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "ps_internal.h"

namespace {

thread_local std::string g_last_error;

size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

}  // namespace

namespace ps {

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_error(cudaError_t e, const char* where) {
    g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return PS_ECUDA;
}

void clear_error() { g_last_error.clear(); }

size_t smem_optin() {
    static thread_local int dev_cached = -1;
    static thread_local int bytes = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != dev_cached) {
        cudaDeviceGetAttribute(&bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        dev_cached = dev;
    }
    return (size_t)bytes;
}

cudaError_t allow_smem(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const auto key = std::make_pair(dev, func);
    std::lock_guard<std::mutex> lock(mu);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) done[key] = bytes;
    return e;
}

int sm_count() {
    static thread_local int dev_cached = -1, sms = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != dev_cached) {
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        dev_cached = dev;
    }
    return sms > 0 ? sms : 148;
}

int validate_scene(const ps_model* m, const ps_scene_view* s) {
    if (!s) return set_error(PS_EINVAL, "scene view is NULL");
    if (s->n_obbs < 0 || s->n_obbs > PS_MAX_OBBS)
        return set_error(PS_EINVAL, "n_obbs out of range [0, " + std::to_string(PS_MAX_OBBS) + "]");
    if (s->n_obbs > 0 && (!s->obb_dims || !s->obb_pose || !s->obb_enable))
        return set_error(PS_EINVAL, "n_obbs > 0 but an OBB array is NULL");
    if (s->n_voxel_layers < 0 || s->n_voxel_layers > PS_MAX_LAYERS)
        return set_error(PS_EINVAL, "n_voxel_layers out of range [0, " + std::to_string(PS_MAX_LAYERS) + "]");
    if (s->n_voxel_layers > 0 &&
        (!s->voxel_params || !s->voxel_pose || !s->voxel_enable || !s->voxel_features || s->max_voxels_per_layer <= 0))
        return set_error(PS_EINVAL, "n_voxel_layers > 0 but a voxel array is NULL or max_voxels_per_layer <= 0");
    if (s->esdf_mode != PS_ESDF_NEAREST && s->esdf_mode != PS_ESDF_TRILINEAR)
        return set_error(PS_EINVAL, "esdf_mode must be PS_ESDF_NEAREST or PS_ESDF_TRILINEAR");
    return check_model_device(m);
}

int check_model_device(const ps_model* m) {
    if (!m) return set_error(PS_EINVAL, "model is NULL");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    if (dev != m->info.device)
        return set_error(PS_EINVAL, "model was created on device " + std::to_string(m->info.device) + " but device " +
                                        std::to_string(dev) +
                                        " is current; make the model's device current (or build one per device)");
    return PS_OK;
}

size_t scene_smem_bytes(const ps_scene_view* s) {
    size_t n = (size_t)std::max(s->n_obbs, 1);
    return align16(n * sizeof(ObbPrep)) + align16(n * sizeof(int)) + sizeof(LayerPrep) * PS_MAX_LAYERS + 64;
}

}  // namespace ps

// ---------------------------------------------------------------------------
// C ABI: model
// ---------------------------------------------------------------------------
namespace {

bool ft_last_row_ok(const float* ft) { return ft[12] == 0.0f && ft[13] == 0.0f && ft[14] == 0.0f && ft[15] == 1.0f; }

}  // namespace

extern "C" const char* ps_last_error(void) { return g_last_error.c_str(); }

extern "C" const char* ps_version(void) { return "prismplan_b200 0.1 (sm_100a)"; }

extern "C" int ps_model_create(const ps_model_desc* d, ps_model** out) {
    PS_NVTX("ps_model_create");
    using namespace ps;
    clear_error();
    if (!d || !out) return set_error(PS_EINVAL, "NULL descriptor or output");
    *out = nullptr;
    const int nj = d->n_joints, nd = d->n_dof, ns = d->n_spheres, na = d->n_approx_spheres;
    if (nj < 1 || nj > PS_MAX_JOINTS) return set_error(PS_EINVAL, "n_joints must be in [1, 20]");
    if (nd < 1 || nd > PS_MAX_DOF) return set_error(PS_EINVAL, "n_dof must be in [1, 14]");
    if (ns < 0 || ns > PS_MAX_SPHERES || na < 0 || na > PS_MAX_SPHERES)
        return set_error(PS_EINVAL, "sphere counts must be in [0, 512]");
    if (!d->fixed_transforms || !d->joint_types) return set_error(PS_EINVAL, "fixed_transforms/joint_types NULL");
    if (ns > 0 && (!d->spheres || !d->sphere_to_joint)) return set_error(PS_EINVAL, "spheres/sphere_to_joint NULL");
    if (na > 0 && (!d->approx_spheres || !d->approx_sphere_to_joint))
        return set_error(PS_EINVAL, "approx spheres NULL");
    if (!d->joint_lower || !d->joint_upper) return set_error(PS_EINVAL, "joint limits NULL");
    const float* aft = d->approx_fixed_transforms ? d->approx_fixed_transforms : d->fixed_transforms;
    const int* atypes = d->approx_joint_types ? d->approx_joint_types : d->joint_types;

    // Tree topology with serial defaults (robot_model.cuh:204-236).
    std::vector<int> parents(nj), id2dof(nj), tmem(nj), dfs(nj);
    for (int i = 0; i < nj; ++i) {
        parents[i] = d->joint_parents ? d->joint_parents[i] : (i > 0 ? i - 1 : 0);
        id2dof[i] = d->joint_id_to_dof ? d->joint_id_to_dof[i] : i - 1;
        tmem[i] = d->t_memory_idx ? d->t_memory_idx[i] : (i == 0 ? 0 : 1);
        dfs[i] = d->dfs_order ? d->dfs_order[i] : i;
    }
    std::vector<int> pos(nj, -1);
    for (int p = 0; p < nj; ++p) {
        if (dfs[p] < 0 || dfs[p] >= nj || pos[dfs[p]] >= 0) return set_error(PS_EINVAL, "dfs_order is not a permutation");
        pos[dfs[p]] = p;
    }
    int n_slots = 1;
    for (int i = 0; i < nj; ++i) {
        if (tmem[i] < 0 || tmem[i] > 1) return set_error(PS_EINVAL, "t_memory_idx must be 0 or 1 (two FK slots)");
        n_slots = std::max(n_slots, tmem[i] + 1);
        if (parents[i] < 0 || parents[i] >= nj) return set_error(PS_EINVAL, "joint_parents out of range");
        if (id2dof[i] < -1 || id2dof[i] >= nd) return set_error(PS_EINVAL, "joint_id_to_dof out of range");
        for (const int* ty : {d->joint_types, atypes})
            if (ty[i] < PS_FIXED || ty[i] > PS_Z_ROT) return set_error(PS_EINVAL, "joint type outside -1..5");
        if (!ft_last_row_ok(d->fixed_transforms + 16 * i) || !ft_last_row_ok(aft + 16 * i))
            return set_error(PS_EINVAL, "fixed transform row 3 must be exactly (0, 0, 0, 1)");
    }
    // Every non-root joint: parent visited earlier, and the parent's slot still
    // holds the parent's frame when the joint is visited (the reference FK
    // overwrites slots in DFS order, runtime_kinematics.cuh:42-71).
    {
        int holder[2] = {dfs[0], dfs[0]};   // both slots start as the root identity
        for (int p = 1; p < nj; ++p) {
            int i = dfs[p], par = parents[i];
            if (pos[par] >= p) return set_error(PS_EINVAL, "dfs_order visits a joint before its parent");
            if (holder[tmem[par]] != par && !(par == dfs[0] && holder[tmem[par]] == dfs[0]))
                return set_error(PS_EINVAL, "t_memory_idx overwrites a parent frame before its child is visited");
            if (d->joint_types[i] != PS_FIXED && id2dof[i] < 0)
                return set_error(PS_EINVAL, "a moving joint has joint_id_to_dof = -1");
            holder[tmem[i]] = i;
        }
    }
    for (int s = 0; s < ns; ++s)
        if (d->sphere_to_joint[s] < 0 || d->sphere_to_joint[s] >= nj) return set_error(PS_EINVAL, "sphere_to_joint out of range");
    for (int a = 0; a < na; ++a)
        if (d->approx_sphere_to_joint[a] < 0 || d->approx_sphere_to_joint[a] >= nj)
            return set_error(PS_EINVAL, "approx_sphere_to_joint out of range");

    // Reorder spheres by the DFS position of their joint, ascending original
    // index within a joint (the CSR order of robot_model.cuh:180-198).
    auto reorder = [&](int n, const int* to_joint, std::vector<int>& order, std::vector<int>& beg,
                       std::vector<int>& end) {
        order.resize(n);
        for (int s = 0; s < n; ++s) order[s] = s;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return pos[to_joint[a]] < pos[to_joint[b]]; });
        beg.assign(nj, 0);
        end.assign(nj, 0);
        int k = 0;
        for (int p = 0; p < nj; ++p) {
            beg[p] = k;
            while (k < n && pos[to_joint[order[k]]] == p) ++k;
            end[p] = k;
        }
    };
    std::vector<int> sorder, sbeg, send, aorder, abeg, aend;
    reorder(ns, d->sphere_to_joint, sorder, sbeg, send);
    reorder(na, d->approx_sphere_to_joint, aorder, abeg, aend);
    std::vector<int> snew(ns), anew(na);
    for (int k = 0; k < ns; ++k) snew[sorder[k]] = k;
    for (int k = 0; k < na; ++k) anew[aorder[k]] = k;

    auto expand = [&](const int* r, int nr, int nsph, const std::vector<int>& remap, std::vector<uint32_t>& out_pairs,
                      const char* what) -> int {
        for (int k = 0; k < nr; ++k) {
            int i = r[3 * k], a = r[3 * k + 1], b = r[3 * k + 2];
            if (i < 0 || i >= nsph || a < 0 || b >= nsph || a > b + 1)
                return set_error(PS_EINVAL, std::string(what) + " range out of bounds");
            for (int j = a; j <= b; ++j) out_pairs.push_back((uint32_t)remap[i] | ((uint32_t)remap[j] << 16));
        }
        return PS_OK;
    };
    std::vector<uint32_t> pairs, apairs;
    if (d->n_self_cc_ranges > 0) {
        if (!d->self_cc_ranges) return set_error(PS_EINVAL, "self_cc_ranges NULL");
        int rc = expand(d->self_cc_ranges, d->n_self_cc_ranges, ns, snew, pairs, "self_cc");
        if (rc) return rc;
    }
    if (d->n_approx_self_cc_ranges > 0) {
        if (!d->approx_self_cc_ranges) return set_error(PS_EINVAL, "approx_self_cc_ranges NULL");
        int rc = expand(d->approx_self_cc_ranges, d->n_approx_self_cc_ranges, na, anew, apairs, "approx_self_cc");
        if (rc) return rc;
    }

    // Self pairs as runs for the prefilters of the self check and the cost
    // kernels: a run is one sphere i against consecutive spheres j0..j0+len-1
    // of one joint q (pairs sorted by (i, q, j), split where j skips).
    // sruns[r] = (i | q << 9 | len << 14, j0).
    std::vector<int> sph_pos(std::max(ns, 1), 0);
    for (int p = 0; p < nj; ++p)
        for (int k = sbeg[p]; k < send[p]; ++k) sph_pos[k] = p;
    std::vector<uint32_t> opairs(pairs);
    std::stable_sort(opairs.begin(), opairs.end(), [&](uint32_t x, uint32_t y) {
        const int xi = x & 0xffff, xj = x >> 16, yi = y & 0xffff, yj = y >> 16;
        if (xi != yi) return xi < yi;
        if (sph_pos[xj] != sph_pos[yj]) return sph_pos[xj] < sph_pos[yj];
        return xj < yj;
    });
    // A run covers consecutive reordered spheres j0, j0 + 1, ... of one joint.
    struct Run {
        int a, q, i;
        uint32_t w0, w1;
    };
    std::vector<Run> runs;
    for (size_t k = 0; k < opairs.size();) {
        const int i = opairs[k] & 0xffff, q = sph_pos[opairs[k] >> 16];
        const int j0 = (int)(opairs[k] >> 16);
        size_t e = k + 1;
        while (e < opairs.size() && (int)(opairs[e] & 0xffff) == i && (int)(opairs[e] >> 16) == j0 + (int)(e - k) &&
               sph_pos[opairs[e] >> 16] == q && e - k < 511)
            ++e;
        runs.push_back({sph_pos[i], q, i, (uint32_t)i | (uint32_t)q << 9 | (uint32_t)(e - k) << 14, (uint32_t)j0});
        k = e;
    }
    if (runs.size() > 65535) return set_error(PS_EINVAL, "too many self-pair runs");
    // Runs ordered by joint pair (joint of i, joint q), then i; the joint-pair
    // table sjp[k] = (a | q << 16, first run, end run, 0) lets the cost
    // kernels cull whole joint pairs by their bound spheres.
    std::stable_sort(runs.begin(), runs.end(), [](const Run& x, const Run& y) {
        if (x.a != y.a) return x.a < y.a;
        if (x.q != y.q) return x.q < y.q;
        return x.i < y.i;
    });
    std::vector<uint32_t> sruns;   // 2 words per run
    std::vector<uint32_t> sjp;     // 4 words per joint pair
    for (size_t r = 0; r < runs.size(); ++r) {
        if (r == 0 || runs[r].a != runs[r - 1].a || runs[r].q != runs[r - 1].q) {
            if (!sjp.empty()) sjp[sjp.size() - 2] = (uint32_t)r;
            sjp.push_back((uint32_t)runs[r].a | (uint32_t)runs[r].q << 16);
            sjp.push_back((uint32_t)r);
            sjp.push_back(0);
            sjp.push_back(0);
        }
        sruns.push_back(runs[r].w0);
        sruns.push_back(runs[r].w1);
    }
    if (!sjp.empty()) sjp[sjp.size() - 2] = (uint32_t)runs.size();
    // The cost kernels visit the joint pairs in this table's order and cull
    // by the smallest clearance found so far, so pairs likely to be close come
    // first: by DFS distance |q - a| (on a chain, the number of joints
    // between them), then (a, q). The runs keep their order, which defines
    // the tie-break among equal clearances.
    {
        const size_t njp = sjp.size() / 4;
        std::vector<size_t> ord(njp);
        for (size_t k = 0; k < njp; ++k) ord[k] = k;
        auto gap = [&](size_t k) {
            const int a = (int)(sjp[4 * k] & 0xffffu), q = (int)(sjp[4 * k] >> 16);
            return a > q ? a - q : q - a;
        };
        std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return gap(x) < gap(y); });
        std::vector<uint32_t> sorted(sjp.size());
        for (size_t k = 0; k < njp; ++k)
            for (int w = 0; w < 4; ++w) sorted[4 * k + w] = sjp[4 * ord[k] + w];
        sjp.swap(sorted);
    }

    bool shares = std::memcmp(aft, d->fixed_transforms, sizeof(float) * 16 * nj) == 0;
    for (int i = 0; i < nj && shares; ++i) shares = atypes[i] == d->joint_types[i];
    // The bound centre of a joint with an approximate sphere is that sphere's
    // centre (fill_joints below); on a shared chain its world position is the
    // approximate sphere's, bit for bit.
    bool bound_from_apx = shares;
    for (int p = 0; p < nj && bound_from_apx; ++p)
        if (send[p] > sbeg[p] && aend[p] <= abeg[p]) bound_from_apx = false;

    // ---- blob layout ----
    BlobHeader h{};
    size_t off = align16(sizeof(BlobHeader));
    h.off_joints = (int)off;
    off += align16(sizeof(JointRec) * nj);
    h.off_apx_joints = (int)off;
    if (!shares) off += align16(sizeof(JointRec) * nj);
    h.off_spheres = (int)off;
    off += align16(sizeof(float4) * std::max(ns, 1));
    h.off_sph_orig = (int)off;
    off += align16(sizeof(int) * std::max(ns, 1));
    h.off_apx = (int)off;
    off += align16(sizeof(float4) * std::max(na, 1));
    h.off_apx_orig = (int)off;
    off += align16(sizeof(int) * std::max(na, 1));
    const size_t core = off;
    const size_t off_pairs = core;
    off += align16(sizeof(uint32_t) * std::max<size_t>(pairs.size(), 1));
    const size_t off_apairs = off;
    off += align16(sizeof(uint32_t) * std::max<size_t>(apairs.size(), 1));
    const size_t off_sruns = off;
    off += align16(sizeof(uint32_t) * std::max<size_t>(sruns.size(), 2));
    const size_t off_sjp = off;
    off += align16(sizeof(uint32_t) * std::max<size_t>(sjp.size(), 4));
    const size_t off_lower = off;
    off += align16(sizeof(float) * nd);
    const size_t off_upper = off;
    off += align16(sizeof(float) * nd);
    const size_t off_status = off;
    off += 16;
    const size_t total = align16(off);

    h.n_dof = nd;
    h.n_joints = nj;
    h.n_spheres = ns;
    h.n_approx = na;
    h.n_self_pairs = (int)pairs.size();
    h.n_apx_self_pairs = (int)apairs.size();
    h.approx_shares_chain = shares ? 1 : 0;
    h.n_t_slots = n_slots;
    h.off_apx = h.off_apx;
    h.bytes_core = (int)core;
    h.bytes_total = (int)total;

    std::vector<unsigned char> host(total, 0);
    std::memcpy(host.data(), &h, sizeof(h));
    int max_js = 0, max_ja = 0;
    auto fill_joints = [&](size_t at, const float* ftab, const int* ttab) {
        JointRec* J = reinterpret_cast<JointRec*>(host.data() + at);
        for (int p = 0; p < nj; ++p) {
            int i = dfs[p];
            for (int k = 0; k < 12; ++k) J[p].ft[k] = ftab[16 * i + k];
            J[p].type = ttab[i];
            J[p].dof = id2dof[i];
            J[p].parent_slot = tmem[parents[i]];
            J[p].slot = tmem[i];
            J[p].sph_beg = sbeg[p];
            J[p].sph_end = send[p];
            J[p].apx_beg = abeg[p];
            J[p].apx_end = aend[p];
            J[p].parent_pos = pos[parents[i]];
            max_js = std::max(max_js, send[p] - sbeg[p]);
            max_ja = std::max(max_ja, aend[p] - abeg[p]);
            // Enclosing sphere (FP64): centre = first approximate sphere, else
            // the centroid of the exact spheres; radius = max |c - ref| + r.
            double cx = 0, cy = 0, cz = 0, R = -1.0;
            if (aend[p] > abeg[p]) {
                const float* a = d->approx_spheres + 4 * aorder[abeg[p]];
                cx = a[0]; cy = a[1]; cz = a[2];
            } else if (send[p] > sbeg[p]) {
                for (int k = sbeg[p]; k < send[p]; ++k) {
                    const float* s = d->spheres + 4 * sorder[k];
                    cx += s[0]; cy += s[1]; cz += s[2];
                }
                double inv = 1.0 / (send[p] - sbeg[p]);
                cx *= inv; cy *= inv; cz *= inv;
            }
            auto grow = [&](const float* s) {
                double dx = s[0] - cx, dy = s[1] - cy, dz = s[2] - cz;
                R = std::max(R, std::sqrt(dx * dx + dy * dy + dz * dz) + (double)s[3]);
            };
            for (int k = sbeg[p]; k < send[p]; ++k) grow(d->spheres + 4 * sorder[k]);
            for (int k = abeg[p]; k < aend[p]; ++k) grow(d->approx_spheres + 4 * aorder[k]);
            J[p].bound = make_float4((float)cx, (float)cy, (float)cz, R < 0 ? -1.0f : (float)(R * (1.0 + 1e-6) + 1e-6));
        }
    };
    fill_joints(h.off_joints, d->fixed_transforms, d->joint_types);
    if (!shares) fill_joints(h.off_apx_joints, aft, atypes);
    float4* S = reinterpret_cast<float4*>(host.data() + h.off_spheres);
    int* SO = reinterpret_cast<int*>(host.data() + h.off_sph_orig);
    for (int k = 0; k < ns; ++k) {
        const float* s = d->spheres + 4 * sorder[k];
        S[k] = make_float4(s[0], s[1], s[2], s[3]);
        SO[k] = sorder[k];
    }
    float4* A = reinterpret_cast<float4*>(host.data() + h.off_apx);
    int* AO = reinterpret_cast<int*>(host.data() + h.off_apx_orig);
    for (int k = 0; k < na; ++k) {
        const float* s = d->approx_spheres + 4 * aorder[k];
        A[k] = make_float4(s[0], s[1], s[2], s[3]);
        AO[k] = aorder[k];
    }
    if (!pairs.empty()) std::memcpy(host.data() + off_pairs, pairs.data(), pairs.size() * 4);
    if (!apairs.empty()) std::memcpy(host.data() + off_apairs, apairs.data(), apairs.size() * 4);
    if (!sruns.empty()) std::memcpy(host.data() + off_sruns, sruns.data(), sruns.size() * 4);
    if (!sjp.empty()) std::memcpy(host.data() + off_sjp, sjp.data(), sjp.size() * 4);
    std::memcpy(host.data() + off_lower, d->joint_lower, sizeof(float) * nd);
    std::memcpy(host.data() + off_upper, d->joint_upper, sizeof(float) * nd);

    ps_model* m = new ps_model();
    cudaError_t e = cudaMalloc(&m->alloc, total);
    if (e != cudaSuccess) {
        delete m;
        return set_error(PS_ENOMEM, std::string("cudaMalloc model: ") + cudaGetErrorString(e));
    }
    e = cudaMemcpy(m->alloc, host.data(), total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(m->alloc);
        delete m;
        return cuda_error(e, "cudaMemcpy model");
    }
    unsigned char* base = reinterpret_cast<unsigned char*>(m->alloc);
    m->alloc_bytes = total;
    m->dev.blob = base;
    m->dev.self_pairs = reinterpret_cast<const uint32_t*>(base + off_pairs);
    m->dev.apx_self_pairs = reinterpret_cast<const uint32_t*>(base + off_apairs);
    m->dev.sruns = reinterpret_cast<const uint2*>(base + off_sruns);
    m->dev.n_sruns = (int)(sruns.size() / 2);
    m->dev.sjp = reinterpret_cast<const uint4*>(base + off_sjp);
    m->dev.n_sjp = (int)(sjp.size() / 4);
    m->dev.bound_from_apx = bound_from_apx ? 1 : 0;
    m->dev.lower = reinterpret_cast<const float*>(base + off_lower);
    m->dev.upper = reinterpret_cast<const float*>(base + off_upper);
    m->dev.status = reinterpret_cast<int*>(base + off_status);
    m->dev.bytes_core = (int)core;
    m->dev.stage_polls = PS_STAGE_POLLS;
    m->max_joint_spheres = max_js;
    m->root_slot_only = tmem[dfs[0]] == 0;
    for (int p = 1; p < nj; ++p) m->root_slot_only = m->root_slot_only && tmem[dfs[p]] == 1;
    m->max_joint_approx = max_ja;
    m->sph_orig = sorder;
    int dev = 0;
    cudaGetDevice(&dev);
    m->info.n_dof = nd;
    m->info.n_joints = nj;
    m->info.n_spheres = ns;
    m->info.n_approx_spheres = na;
    m->info.n_self_pairs = (int)pairs.size();
    m->info.n_approx_self_pairs = (int)apairs.size();
    m->info.n_t_slots = n_slots;
    m->info.approx_shares_chain = shares ? 1 : 0;
    m->info.device = dev;
    m->info.device_bytes = total;
    *out = m;
    return PS_OK;
}

extern "C" int ps_model_destroy(ps_model* m) {
    if (!m) return PS_OK;
    if (m->alloc) cudaFree(m->alloc);
    delete m;
    return PS_OK;
}

extern "C" int ps_model_set_limits(ps_model* m, const float* lower, const float* upper) {
    ps::clear_error();
    if (!m || !lower || !upper) return ps::set_error(PS_EINVAL, "NULL argument");
    PS_TRY_CUDA(cudaMemcpy((void*)m->dev.lower, lower, sizeof(float) * m->info.n_dof, cudaMemcpyHostToDevice));
    PS_TRY_CUDA(cudaMemcpy((void*)m->dev.upper, upper, sizeof(float) * m->info.n_dof, cudaMemcpyHostToDevice));
    return PS_OK;
}

extern "C" int ps_model_get_info(const ps_model* m, ps_model_info* info) {
    if (!m || !info) return ps::set_error(PS_EINVAL, "NULL argument");
    *info = m->info;
    return PS_OK;
}

extern "C" int ps_model_set_wait_limit(ps_model* m, int polls) {
    ps::clear_error();
    if (!m) return ps::set_error(PS_EINVAL, "model is NULL");
    m->dev.stage_polls = polls < 0 ? PS_STAGE_POLLS : polls;
    return PS_OK;
}

extern "C" int ps_model_poll_status(ps_model* m, int* code) {
    ps::clear_error();
    if (!m || !code) return ps::set_error(PS_EINVAL, "NULL argument");
    int v = 0;
    PS_TRY_CUDA(cudaMemcpy(&v, m->dev.status, sizeof(int), cudaMemcpyDeviceToHost));
    *code = v;
    if (v != 0) {
        int z = 0;
        PS_TRY_CUDA(cudaMemcpy(m->dev.status, &z, sizeof(int), cudaMemcpyHostToDevice));
    }
    return PS_OK;
}
