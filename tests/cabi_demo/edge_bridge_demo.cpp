// edge_bridge_demo.cpp -- a C++ caller of the C ABI, the way the reference's
// C++ planners hold EdgeEvalGpu (code/gpu_planning/cpp/src/planning/
// edge_batch_bridge.hh:27-111): build the robot model from descriptor arrays,
// bind a scene of device OBB arrays (SceneCollisionData layout), create the
// host-buffer edge bridge and evaluate host edges twice (the second call
// replays the captured graph). No Python, no torch.
//
// usage: edge_bridge_demo <problem file> <output file>
// The problem file (written by tests/test_gpu_cabi_cpp.py) holds, little
// endian: int32 magic 0x50534231; int32 n_dof, n_joints, n_spheres,
// n_self_ranges, n_approx, n_approx_ranges, has_tree, n_obbs, n_edges,
// max_samples; float32 max_joint_step; then the descriptor arrays in
// ps_model_desc order (the four tree arrays only when has_tree), the OBB
// arrays (dims [n][4], inverse pose [n][8], enable [n] bytes padded to 4)
// and the edges (from, to: [n_edges][n_dof]). The output file gets
// valid [n_edges] bytes then cost [n_edges] float32, from the second call.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "prism_b200.h"

namespace {

struct Reader {
    std::vector<unsigned char> buf;
    size_t pos = 0;
    bool ok = true;
    template <class T>
    std::vector<T> take(size_t n) {
        std::vector<T> v(n);
        const size_t bytes = n * sizeof(T);
        if (pos + bytes > buf.size()) {
            ok = false;
            return v;
        }
        if (bytes) std::memcpy(v.data(), buf.data() + pos, bytes);
        pos += bytes;
        return v;
    }
    int32_t i32() { return take<int32_t>(1)[0]; }
};

int fail(const char* what, int rc) {
    std::fprintf(stderr, "%s failed: status %d: %s\n", what, rc, ps_last_error());
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <problem file> <output file>\n", argv[0]);
        return 2;
    }
    Reader r;
    {
        FILE* f = std::fopen(argv[1], "rb");
        if (!f) return 2;
        std::fseek(f, 0, SEEK_END);
        r.buf.resize((size_t)std::ftell(f));
        std::fseek(f, 0, SEEK_SET);
        const size_t got = std::fread(r.buf.data(), 1, r.buf.size(), f);
        std::fclose(f);
        if (got != r.buf.size()) return 2;
    }
    if (r.i32() != 0x50534231) return 2;
    const int D = r.i32(), NJ = r.i32(), NS = r.i32(), NR = r.i32(), NA = r.i32(), NAR = r.i32();
    const int has_tree = r.i32(), NO = r.i32(), E = r.i32(), max_samples = r.i32();
    const float step = r.take<float>(1)[0];
    auto ft = r.take<float>((size_t)NJ * 16);
    auto jt = r.take<int32_t>(NJ);
    auto sp = r.take<float>((size_t)NS * 4);
    auto s2j = r.take<int32_t>(NS);
    auto rng = r.take<int32_t>((size_t)NR * 3);
    auto ap = r.take<float>((size_t)NA * 4);
    auto a2j = r.take<int32_t>(NA);
    auto arng = r.take<int32_t>((size_t)NAR * 3);
    auto lo = r.take<float>(D), hi = r.take<float>(D);
    std::vector<int32_t> par, j2d, tmi, dfs;
    if (has_tree) {
        par = r.take<int32_t>(NJ);
        j2d = r.take<int32_t>(NJ);
        tmi = r.take<int32_t>(NJ);
        dfs = r.take<int32_t>(NJ);
    }
    auto dims = r.take<float>((size_t)NO * 4);
    auto pose = r.take<float>((size_t)NO * 8);
    auto en = r.take<uint8_t>(((size_t)NO + 3) & ~size_t(3));
    auto from = r.take<float>((size_t)E * D), to = r.take<float>((size_t)E * D);
    if (!r.ok) return 2;

    ps_model_desc d;
    std::memset(&d, 0, sizeof(d));
    d.n_dof = D;
    d.n_joints = NJ;
    d.fixed_transforms = ft.data();
    d.joint_types = jt.data();
    d.n_spheres = NS;
    d.spheres = sp.data();
    d.sphere_to_joint = s2j.data();
    d.n_self_cc_ranges = NR;
    d.self_cc_ranges = NR ? rng.data() : nullptr;
    d.n_approx_spheres = NA;
    d.approx_spheres = NA ? ap.data() : nullptr;
    d.approx_sphere_to_joint = NA ? a2j.data() : nullptr;
    d.n_approx_self_cc_ranges = NAR;
    d.approx_self_cc_ranges = NAR ? arng.data() : nullptr;
    d.joint_lower = lo.data();
    d.joint_upper = hi.data();
    if (has_tree) {
        d.joint_parents = par.data();
        d.joint_id_to_dof = j2d.data();
        d.t_memory_idx = tmi.data();
        d.dfs_order = dfs.data();
    }
    ps_model* model = nullptr;
    if (int rc = ps_model_create(&d, &model)) return fail("ps_model_create", rc);

    // the scene: device arrays in the SceneCollisionData layout, bound without a copy
    float *d_dims = nullptr, *d_pose = nullptr;
    uint8_t* d_en = nullptr;
    if (cudaMalloc(&d_dims, dims.size() * 4 + 16) != cudaSuccess || cudaMalloc(&d_pose, pose.size() * 4 + 16) != cudaSuccess ||
        cudaMalloc(&d_en, en.size() + 16) != cudaSuccess)
        return 3;
    cudaMemcpy(d_dims, dims.data(), dims.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_pose, pose.data(), pose.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_en, en.data(), en.size(), cudaMemcpyHostToDevice);
    ps_scene_view view;
    std::memset(&view, 0, sizeof(view));
    view.obb_dims = d_dims;
    view.obb_pose = d_pose;
    view.obb_enable = d_en;
    view.n_obbs = NO;
    view.esdf_mode = PS_ESDF_NEAREST;

    ps_edge_bridge* bridge = nullptr;
    if (int rc = ps_edge_bridge_create(model, &view, D, E, &bridge)) return fail("ps_edge_bridge_create", rc);
    ps_edge_params p;
    std::memset(&p, 0, sizeof(p));
    p.granularity = 16;
    p.max_joint_step = step;
    p.max_samples = max_samples;
    std::vector<uint8_t> valid(E);
    std::vector<float> cost(E);
    for (int call = 0; call < 2; ++call)   // the second call replays the captured graph
        if (int rc = ps_edge_bridge_evaluate(bridge, from.data(), to.data(), E, &p, valid.data(), cost.data(), nullptr))
            return fail("ps_edge_bridge_evaluate", rc);
    int status = -1;
    if (int rc = ps_edge_bridge_status(bridge, &status)) return fail("ps_edge_bridge_status", rc);
    if (status != PS_OK) return fail("edge bridge status", status);
    ps_edge_bridge_destroy(bridge);
    ps_model_destroy(model);
    cudaFree(d_dims);
    cudaFree(d_pose);
    cudaFree(d_en);

    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    std::fwrite(valid.data(), 1, valid.size(), o);
    std::fwrite(cost.data(), 4, cost.size(), o);
    std::fclose(o);
    int n_valid = 0;
    for (uint8_t v : valid) n_valid += v;
    std::printf("%d edges, %d valid\n", E, n_valid);
    return 0;
}
