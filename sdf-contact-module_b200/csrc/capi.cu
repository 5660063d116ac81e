// extern "C" entry points for builds, queries and contact (see include/sdfo.h).
#include <cmath>
#include <cstring>

#include "sdfo_internal.cuh"

using namespace sdfo;

namespace {

void check_grid(const sdfo_grid* g)
{
    SDFO_REQUIRE(g != nullptr, SDFO_ERR_INVALID_ARGUMENT, "grid is NULL");
    SDFO_REQUIRE(g->stored_voxels > 0 || g->info.layout == SDFO_LAYOUT_SPARSE,
                 SDFO_ERR_INVALID_ARGUMENT, "grid is empty");
}

void check_mesh(const double* verts, int64_t nv, const int32_t* tris, int64_t nt)
{
    SDFO_REQUIRE(nv > 0 && nt > 0 && verts && tris, SDFO_ERR_EMPTY_MESH,
                 "Empty mesh provided to SdfBuilder");
    SDFO_REQUIRE(nt < (int64_t(1) << 31) && nv < (int64_t(1) << 31), SDFO_ERR_INVALID_ARGUMENT,
                 "mesh too large");
    for (int64_t i = 0; i < 3 * nt; ++i)
        SDFO_REQUIRE(tris[i] >= 0 && tris[i] < nv, SDFO_ERR_INVALID_ARGUMENT,
                     "triangle references invalid vertex");
    for (int64_t i = 0; i < 3 * nv; ++i)
        SDFO_REQUIRE(std::isfinite(verts[i]), SDFO_ERR_INVALID_ARGUMENT,
                     "vertex coordinates must be finite");
}

void check_build_params(const sdfo_build_params* p)
{
    SDFO_REQUIRE(p != nullptr, SDFO_ERR_INVALID_ARGUMENT, "build params are NULL");
    SDFO_REQUIRE(p->max_resolution > 0, SDFO_ERR_INVALID_ARGUMENT, "maxResolution must be positive");
    SDFO_REQUIRE(p->voxel_size > 0.0 || p->target_resolution > 0, SDFO_ERR_INVALID_ARGUMENT,
                 "targetResolution must be positive when voxelSize is 0");
    SDFO_REQUIRE(std::isfinite(p->padding) && std::isfinite(p->voxel_size),
                 SDFO_ERR_INVALID_ARGUMENT, "padding and voxelSize must be finite");
}

} // namespace

extern "C" {

const char* sdfo_version(void) { return "sdfo-b200 0.1.0 (SDFO format 0.1.0)"; }

int sdfo_abi_version(void) { return SDFO_ABI_VERSION; }

int sdfo_device_check(int device)
{
    return guarded([&] {
        int count = 0;
        const cudaError_t e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess || count == 0)
        {
            (void)cudaGetLastError();
            throw Error(SDFO_ERR_NO_DEVICE, "no CUDA device available");
        }
        SDFO_REQUIRE(device >= 0 && device < count, SDFO_ERR_NO_DEVICE, "device index out of range");
        cudaDeviceProp prop;
        SDFO_CUDA(cudaGetDeviceProperties(&prop, device));
        SDFO_REQUIRE(prop.major == 10, SDFO_ERR_NO_DEVICE,
                     std::string("libsdfo_cuda is built for sm_100a; device is ") + prop.name);
    });
}

void sdfo_build_params_default(sdfo_build_params* p)
{
    if (!p) return;
    p->padding = 0.1;
    p->voxel_size = 0.0;
    p->target_resolution = 128;
    p->max_resolution = 512;
}

void sdfo_sparse_build_params_default(sdfo_sparse_build_params* p)
{
    if (!p) return;
    sdfo_build_params_default(&p->base);
    p->block_dim = 8;
    p->halo_voxels = 2;
    p->band_voxels = 8;
    p->store_hessian = 1;
    p->band_distance = 0.0;
}

void sdfo_contact_aware_params_default(sdfo_contact_aware_params* p)
{
    if (!p) return;
    sdfo_build_params_default(&p->base);
    p->max_candidates = 4;
    p->tile_dim = 8;
    p->use_tile_acceleration = 1;
    p->store_hessian = 1;
    p->feature_distance_tolerance = 0.0;
    p->normal_merge_angle_degrees = 5.0;
    p->sparse = 0;
    p->block_dim = 8;
    p->halo_voxels = 2;
    p->band_voxels = 8;
    p->band_distance = 0.0;
}

int sdfo_setup_grid(const double* h_verts, int64_t nv, const sdfo_build_params* p,
                    sdfo_grid_info* out)
{
    return guarded([&] {
        SDFO_REQUIRE(out != nullptr, SDFO_ERR_INVALID_ARGUMENT, "out is NULL");
        SDFO_REQUIRE(h_verts && nv > 0, SDFO_ERR_EMPTY_MESH, "Empty mesh provided to SdfBuilder");
        check_build_params(p);
        *out = setup_grid(h_verts, nv, *p);
    });
}

int sdfo_grid_build_dense(const double* h_verts, int64_t nv, const int32_t* h_tris, int64_t nt,
                          const sdfo_build_params* p, void* stream, sdfo_grid** out)
{
    return guarded([&] {
        SDFO_REQUIRE(out != nullptr, SDFO_ERR_INVALID_ARGUMENT, "out is NULL");
        *out = nullptr;
        check_mesh(h_verts, nv, h_tris, nt);
        check_build_params(p);
        *out = build_dense(h_verts, nv, h_tris, nt, *p, as_stream(stream));
    });
}

int sdfo_device_cache(int64_t limit, int64_t* held)
{
    return guarded([&] { device_cache_control(limit, held); });
}

int sdfo_build_traversal_stats(const double* h_verts, int64_t nv, const int32_t* h_tris, int64_t nt,
                               const sdfo_build_params* p, void* stream, sdfo_traversal_stats* out)
{
    return guarded([&] {
        SDFO_REQUIRE(out != nullptr, SDFO_ERR_INVALID_ARGUMENT, "out is NULL");
        std::memset(out, 0, sizeof(*out));
        check_mesh(h_verts, nv, h_tris, nt);
        check_build_params(p);
        count_dense_traversal(h_verts, nv, h_tris, nt, *p, as_stream(stream), out);
    });
}

int sdfo_grid_build_sparse(const double* h_verts, int64_t nv, const int32_t* h_tris, int64_t nt,
                           const sdfo_sparse_build_params* p, void* stream, sdfo_grid** out)
{
    return guarded([&] {
        SDFO_REQUIRE(out != nullptr, SDFO_ERR_INVALID_ARGUMENT, "out is NULL");
        *out = nullptr;
        check_mesh(h_verts, nv, h_tris, nt);
        SDFO_REQUIRE(p != nullptr, SDFO_ERR_INVALID_ARGUMENT, "build params are NULL");
        check_build_params(&p->base);
        SDFO_REQUIRE(p->block_dim > 0, SDFO_ERR_INVALID_ARGUMENT,
                     "Sparse SDF blockDim must be positive");
        SDFO_REQUIRE(p->block_dim <= 16, SDFO_ERR_UNSUPPORTED, "blockDim above 16 is not provided");
        *out = build_sparse(h_verts, nv, h_tris, nt, *p, as_stream(stream));
    });
}

int sdfo_grid_build_contact_aware(const double* h_verts, int64_t nv, const int32_t* h_tris,
                                  int64_t nt, const double* h_corner_normals,
                                  const sdfo_contact_aware_params* p, void* stream,
                                  sdfo_grid** out)
{
    return guarded([&] {
        SDFO_REQUIRE(out != nullptr, SDFO_ERR_INVALID_ARGUMENT, "out is NULL");
        *out = nullptr;
        SDFO_REQUIRE(p != nullptr, SDFO_ERR_INVALID_ARGUMENT, "build params are NULL");
        // SdfBuilder.cpp:419-425 / 554-562
        SDFO_REQUIRE(nv > 0 && nt > 0 && h_verts && h_tris, SDFO_ERR_EMPTY_MESH,
                     p->sparse ? "Empty mesh provided to sparse contact-aware SdfBuilder"
                               : "Empty mesh provided to contact-aware SdfBuilder");
        SDFO_REQUIRE(h_corner_normals != nullptr, SDFO_ERR_INVALID_ARGUMENT,
                     p->sparse ? "Sparse contact-aware SDF requires one corner-normal triplet per triangle"
                               : "Contact-aware SDF requires one corner-normal triplet per triangle");
        SDFO_REQUIRE(p->max_candidates > 0, SDFO_ERR_INVALID_ARGUMENT,
                     p->sparse ? "Sparse contact-aware SDF maxCandidates must be positive"
                               : "Contact-aware SDF maxCandidates must be positive");
        SDFO_REQUIRE(!p->sparse || p->block_dim > 0, SDFO_ERR_INVALID_ARGUMENT,
                     "Sparse contact-aware SDF blockDim must be positive");
        SDFO_REQUIRE(!p->sparse || p->block_dim <= 16, SDFO_ERR_UNSUPPORTED,
                     "blockDim above 16 is not provided");
        check_mesh(h_verts, nv, h_tris, nt);
        check_build_params(&p->base);
        *out = build_contact_aware(h_verts, nv, h_tris, nt, h_corner_normals, *p, as_stream(stream));
    });
}

int sdfo_grid_build_sparse_batched(const sdfo_mesh_desc* meshes, int32_t n, void* stream,
                                   sdfo_grid** out)
{
    return guarded([&] {
        SDFO_REQUIRE(out != nullptr && meshes != nullptr, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        SDFO_REQUIRE(n > 0, SDFO_ERR_INVALID_ARGUMENT, "batched build needs at least one mesh");
        for (int32_t m = 0; m < n; ++m) out[m] = nullptr;
        for (int32_t m = 0; m < n; ++m)
        {
            const sdfo_mesh_desc& d = meshes[m];
            check_mesh(d.h_verts, d.nv, d.h_tris, d.nt);
            check_build_params(&d.params.base);
            SDFO_REQUIRE(d.params.block_dim > 0, SDFO_ERR_INVALID_ARGUMENT,
                         "Sparse SDF blockDim must be positive");
            SDFO_REQUIRE(d.params.block_dim <= 16, SDFO_ERR_UNSUPPORTED,
                         "blockDim above 16 is not provided");
        }
        const std::vector<sdfo_grid*> grids = build_sparse_batched(meshes, n, as_stream(stream));
        for (int32_t m = 0; m < n; ++m) out[m] = grids[(size_t)m];
    });
}

int sdfo_set_fill_ctas_per_sm(int32_t ctas)
{
    return guarded([&] {
        SDFO_REQUIRE(ctas >= 0 && ctas <= 64, SDFO_ERR_INVALID_ARGUMENT, "CTAs per SM out of range");
        set_fill_ctas_per_sm(ctas);
    });
}

int sdfo_set_bvh_mode(int32_t mode)
{
    return guarded([&] {
        SDFO_REQUIRE(mode == SDFO_BVH_REFERENCE || mode == SDFO_BVH_LBVH, SDFO_ERR_INVALID_ARGUMENT,
                     "unknown BVH mode");
        set_bvh_mode(mode);
    });
}

int sdfo_get_bvh_mode(void) { return bvh_mode(); }

int sdfo_set_sign_mode(int32_t mode)
{
    return guarded([&] {
        SDFO_REQUIRE(mode == SDFO_SIGN_RAY_PARITY || mode == SDFO_SIGN_PSEUDONORMAL, SDFO_ERR_INVALID_ARGUMENT,
                     "unknown sign mode");
        set_sign_mode(mode);
    });
}

int sdfo_get_sign_mode(void) { return sign_mode(); }

int sdfo_query(const sdfo_grid* g, int32_t mode, const void* d_points, int32_t points_f64,
               int64_t n, float* d_gap, float* d_grad, float* d_unit, float* d_witness,
               uint8_t* d_valid, float* d_hess, void* stream)
{
    return guarded([&] {
        check_grid(g);
        SDFO_REQUIRE(n >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative query count");
        if (n == 0) return;
        SDFO_REQUIRE(d_points && d_gap, SDFO_ERR_INVALID_ARGUMENT, "points and gap are required");
        SDFO_REQUIRE(mode >= SDFO_FIRST_ORDER && mode <= SDFO_CONTACT_AWARE,
                     SDFO_ERR_INVALID_ARGUMENT, "unknown query mode");
        SDFO_REQUIRE(n <= (int64_t)65535 * 256 * 4096, SDFO_ERR_INVALID_ARGUMENT, "too many queries");
        const QueryOutputs o{d_gap, d_grad, d_unit, d_witness, d_valid, d_hess};
        launch_query(make_view(g), mode, d_points, points_f64 != 0, n, o, as_stream(stream));
    });
}

int sdfo_query_backward(const sdfo_grid* g, int32_t mode, const float* d_points, int64_t n,
                        const float* d_dgap, const float* d_dgrad, float* d_dpoints,
                        float* d_dgrid, void* stream)
{
    return guarded([&] {
        check_grid(g);
        SDFO_REQUIRE(n >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative query count");
        if (n == 0) return;
        SDFO_REQUIRE(d_points != nullptr, SDFO_ERR_INVALID_ARGUMENT, "points are required");
        SDFO_REQUIRE(mode == SDFO_TRILINEAR || mode == SDFO_TRICUBIC, SDFO_ERR_UNSUPPORTED,
                     "query backward supports Trilinear and Tricubic");
        SDFO_REQUIRE((reinterpret_cast<uintptr_t>(d_dgrid) & 15) == 0, SDFO_ERR_INVALID_ARGUMENT,
                     "grid gradient buffer must be 16-byte aligned");
        launch_query_backward(make_view(g), mode, d_points, n, d_dgap, d_dgrad, d_dpoints, d_dgrid,
                              as_stream(stream));
    });
}

int sdfo_query_candidates(const sdfo_grid* g, int32_t mode, const float* d_points, int64_t n,
                          float* d_gap, float* d_normal, float* d_witness, uint8_t* d_valid,
                          int32_t* d_ncand, float* d_kgap, float* d_knormal, float* d_kwitness,
                          int32_t* d_kbranch, void* stream)
{
    return guarded([&] {
        check_grid(g);
        SDFO_REQUIRE(n >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative query count");
        if (n == 0) return;
        SDFO_REQUIRE(d_points && d_gap && d_normal && d_witness && d_valid && d_ncand && d_kgap &&
                         d_knormal && d_kwitness && d_kbranch,
                     SDFO_ERR_INVALID_ARGUMENT, "every output of sdfo_query_candidates is required");
        SDFO_REQUIRE(mode >= SDFO_FIRST_ORDER && mode <= SDFO_CONTACT_AWARE,
                     SDFO_ERR_INVALID_ARGUMENT, "unknown query mode");
        SDFO_REQUIRE(n <= (int64_t)65535 * 256 * 4096, SDFO_ERR_INVALID_ARGUMENT, "too many queries");
        const GridView v = make_view(g);
        const CandidateOutputs co{d_ncand, d_kgap, d_knormal, d_kwitness, d_kbranch};
        const QueryOutputs o{d_gap, nullptr, d_normal, d_witness, d_valid, nullptr};
        cudaStream_t s = as_stream(stream);
        if (mode == SDFO_CONTACT_AWARE && v.ca_stride > 0)
        {
            launch_query_ca(v, d_points, false, n, o, co, s);
            return;
        }
        launch_query(v, mode, d_points, false, n, o, s);
        launch_single_candidate(n, d_gap, d_normal, d_witness, d_valid, co, s);
    });
}

int sdfo_query_candidates_host(const sdfo_grid* g, int32_t mode, const void* h_points,
                               int32_t points_f64, int64_t n, float* h_gap, float* h_normal,
                               float* h_witness, uint8_t* h_valid, int32_t* h_ncand,
                               float* h_kgap, float* h_knormal, float* h_kwitness,
                               int32_t* h_kbranch, void* stream)
{
    return guarded([&] {
        check_grid(g);
        SDFO_REQUIRE(n >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative query count");
        if (n == 0) return;
        SDFO_REQUIRE(h_points && h_gap && h_normal && h_witness && h_valid && h_ncand && h_kgap &&
                         h_knormal && h_kwitness && h_kbranch,
                     SDFO_ERR_INVALID_ARGUMENT, "every output of sdfo_query_candidates_host is required");
        SDFO_REQUIRE(mode >= SDFO_FIRST_ORDER && mode <= SDFO_CONTACT_AWARE,
                     SDFO_ERR_INVALID_ARGUMENT, "unknown query mode");
        SDFO_REQUIRE(n <= (int64_t)65535 * 256 * 4096, SDFO_ERR_INVALID_ARGUMENT, "too many queries");
        cudaStream_t s = as_stream(stream);
        auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
        const size_t N = (size_t)n;
        const size_t pb = N * 3 * (points_f64 ? sizeof(double) : sizeof(float));
        // points | gap | normal | witness | valid | ncand | kgap | knormal | kwitness | kbranch
        const size_t sizes[10] = {pb, 4 * N, 12 * N, 12 * N, N, 4 * N, 32 * N, 96 * N, 96 * N, 32 * N};
        size_t need = 0;
        for (size_t b : sizes) need += up(b);
        std::lock_guard<std::mutex> lock(g->ws_mutex);
        if (g->ws_bytes < need)
        {
            SDFO_CUDA(cudaStreamSynchronize(s));
            device_free(g->ws);
            g->ws = nullptr;
            g->ws_bytes = 0;
            g->ws = device_alloc(need);
            g->ws_bytes = need;
        }
        unsigned char* base = static_cast<unsigned char*>(g->ws);
        unsigned char* d[10];
        for (int i = 0; i < 10; ++i)
        {
            d[i] = base;
            base += up(sizes[i]);
        }
        SDFO_CUDA(cudaMemcpyAsync(d[0], h_points, pb, cudaMemcpyHostToDevice, s));
        float* gap = reinterpret_cast<float*>(d[1]);
        float* nrm = reinterpret_cast<float*>(d[2]);
        float* wit = reinterpret_cast<float*>(d[3]);
        uint8_t* valid = d[4];
        const CandidateOutputs co{reinterpret_cast<int32_t*>(d[5]), reinterpret_cast<float*>(d[6]),
                                  reinterpret_cast<float*>(d[7]), reinterpret_cast<float*>(d[8]),
                                  reinterpret_cast<int32_t*>(d[9])};
        const QueryOutputs o{gap, nullptr, nrm, wit, valid, nullptr};
        const GridView v = make_view(g);
        if (mode == SDFO_CONTACT_AWARE && v.ca_stride > 0)
        {
            launch_query_ca(v, d[0], points_f64 != 0, n, o, co, s);
        }
        else
        {
            launch_query(v, mode, d[0], points_f64 != 0, n, o, s);
            launch_single_candidate(n, gap, nrm, wit, valid, co, s);
        }
        void* outs[9] = {h_gap, h_normal, h_witness, h_valid, h_ncand, h_kgap, h_knormal, h_kwitness,
                         h_kbranch};
        for (int i = 0; i < 9; ++i)
            SDFO_CUDA(cudaMemcpyAsync(outs[i], d[i + 1], sizes[i + 1], cudaMemcpyDeviceToHost, s));
        SDFO_CUDA(cudaStreamSynchronize(s));
    });
}

int sdfo_query_linearize(const sdfo_grid* g, int32_t mode, const float* d_points, int64_t n,
                         float* d_gap, float* d_grad, uint8_t* d_valid, float* d_hess6,
                         void* stream)
{
    return guarded([&] {
        check_grid(g);
        SDFO_REQUIRE(n >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative query count");
        if (n == 0) return;
        SDFO_REQUIRE(mode == SDFO_TRILINEAR || mode == SDFO_TRICUBIC, SDFO_ERR_UNSUPPORTED,
                     "query linearisation supports Trilinear and Tricubic");
        SDFO_REQUIRE(d_points && d_gap && d_grad && d_valid && d_hess6, SDFO_ERR_INVALID_ARGUMENT,
                     "points, gap, grad, valid and hess6 are required");
        SDFO_REQUIRE(n <= (int64_t)65535 * 256 * 4096, SDFO_ERR_INVALID_ARGUMENT, "too many queries");
        QueryOutputs o{d_gap, d_grad, nullptr, nullptr, d_valid, nullptr};
        o.hess6 = d_hess6;
        launch_query(make_view(g), mode, d_points, false, n, o, as_stream(stream));
    });
}

int sdfo_query_backward_saved(const sdfo_grid* g, int32_t mode, const float* d_points, int64_t n,
                              const float* d_grad, const float* d_hess6, const uint8_t* d_valid,
                              const float* d_dgap, const float* d_dgrad, float* d_dpoints,
                              float* d_dgrid, void* stream)
{
    return guarded([&] {
        check_grid(g);
        SDFO_REQUIRE(n >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative query count");
        if (n == 0) return;
        SDFO_REQUIRE(mode == SDFO_TRILINEAR || mode == SDFO_TRICUBIC, SDFO_ERR_UNSUPPORTED,
                     "query backward supports Trilinear and Tricubic");
        SDFO_REQUIRE(d_dpoints == nullptr || (d_grad && d_hess6), SDFO_ERR_INVALID_ARGUMENT,
                     "point gradients need the saved grad and hess6");
        SDFO_REQUIRE(d_dgrid == nullptr || (d_points && d_valid), SDFO_ERR_INVALID_ARGUMENT,
                     "grid gradients need the points and the saved valid flags");
        SDFO_REQUIRE((reinterpret_cast<uintptr_t>(d_dgrid) & 15) == 0, SDFO_ERR_INVALID_ARGUMENT,
                     "grid gradient buffer must be 16-byte aligned");
        SDFO_REQUIRE(n <= (int64_t)65535 * 256 * 4096, SDFO_ERR_INVALID_ARGUMENT, "too many queries");
        const SavedBackward b{d_points, n, d_grad, d_hess6, d_valid, d_dgap, d_dgrad, d_dpoints,
                              d_dgrid};
        launch_backward_saved(make_view(g), mode, b, as_stream(stream));
    });
}

int sdfo_contact_eval(const sdfo_grid* g, int32_t mode, const float* d_quad_x,
                      const float* d_quad_w, int64_t nq, const sdfo_body_state* d_pose_a,
                      int64_t np, const sdfo_body_state* d_body_b,
                      const sdfo_contact_params* h_params, double* d_ft, double* d_jac,
                      void* stream)
{
    return guarded([&] {
        check_grid(g);
        SDFO_REQUIRE(h_params != nullptr, SDFO_ERR_INVALID_ARGUMENT, "contact params are NULL");
        SDFO_REQUIRE(mode == SDFO_TRILINEAR || mode == SDFO_TRICUBIC, SDFO_ERR_UNSUPPORTED,
                     "contact supports Trilinear and Tricubic");
        SDFO_REQUIRE(nq >= 0 && np >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative count");
        if (np == 0) return;
        SDFO_REQUIRE(d_pose_a && d_body_b && d_ft, SDFO_ERR_INVALID_ARGUMENT,
                     "poses, body B and the force output are required");
        SDFO_REQUIRE(nq == 0 || (d_quad_x && d_quad_w), SDFO_ERR_INVALID_ARGUMENT,
                     "quadrature points and weights are required");
        SDFO_REQUIRE(np <= 0x7fffffff && nq <= 0x7fffffff, SDFO_ERR_INVALID_ARGUMENT,
                     "too many poses or points");
        launch_contact(make_view(g), mode, d_quad_x, d_quad_w, nq, d_pose_a, np, d_body_b,
                       *h_params, d_ft, d_jac, as_stream(stream));
    });
}

} // extern "C"
