// Contact pairs: SDFContactEngine.register_pair (prototype/src/dynamics/
// contacts_sdf.py:52-62) -- weights normalised to sum 1 and the AABB_BVH
// point hierarchy of prototype/src/geometry/bvh.py:16-60 built over the
// quadrature points -- and the culled evaluate / measure_pair launches over
// it (the kernels are in contact.cu).
//
// The hierarchy is built on the host exactly as AABB_BVH._build does it:
// box of the node's points, leaf when at most leaf_size points, otherwise a
// split of the longest axis (first on ties) at the box's midpoint, points
// <= mid to the left in their current order; if one side would be empty (all
// points coincide along that axis) a median split of the points sorted along
// the axis (a stable sort here; numpy's default sort does not promise an
// order among equal keys, which only matters for coincident points).  Leaves
// are stored in the order AABB_BVH.query's stack visits them (right child
// first), their points leaf by leaf, so that a query's concatenated index
// list is the kept leaves' points in stored order.
#include <algorithm>
#include <cmath>
#include <memory>
#include <numeric>
#include <vector>

#include "sdfo_internal.cuh"

sdfo_contact_pair::~sdfo_contact_pair()
{
    sdfo::device_free(px);
    sdfo::device_free(pw);
    sdfo::device_free(px64);
    sdfo::device_free(pw64);
    sdfo::device_free(ox64);
    sdfo::device_free(ow64);
    sdfo::device_free(porig);
    sdfo::device_free(pleaf);
    sdfo::device_free(leaf_start);
    sdfo::device_free(leaf_box);
}

namespace sdfo {
namespace {

struct Leaf
{
    std::vector<int32_t> idx;
    double box[6];
};

void box_of(const double* X, const std::vector<int32_t>& idx, double box[6])
{
    for (int a = 0; a < 3; ++a)
    {
        box[a] = INFINITY;
        box[3 + a] = -INFINITY;
    }
    for (int32_t i : idx)
        for (int a = 0; a < 3; ++a)
        {
            const double v = X[3 * (int64_t)i + a];
            box[a] = std::min(box[a], v);
            box[3 + a] = std::max(box[3 + a], v);
        }
}

// AABB_BVH._build (bvh.py:27-60); appends the leaves right subtree first.
void build_node(const double* X, std::vector<int32_t> idx, int leaf_size, std::vector<Leaf>& out)
{
    double box[6];
    box_of(X, idx, box);
    if ((int)idx.size() <= leaf_size)
    {
        Leaf l;
        l.idx = std::move(idx);
        std::copy(box, box + 6, l.box);
        out.push_back(std::move(l));
        return;
    }
    int axis = 0;
    double ext = box[3] - box[0];
    for (int a = 1; a < 3; ++a)
        if (box[3 + a] - box[a] > ext)
        {
            ext = box[3 + a] - box[a];
            axis = a;
        }
    const double mid = (box[axis] + box[3 + axis]) * 0.5;
    std::vector<int32_t> left, right;
    for (int32_t i : idx) (X[3 * (int64_t)i + axis] <= mid ? left : right).push_back(i);
    if (left.empty() || right.empty())
    {
        std::vector<int32_t> order(idx.size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
            return X[3 * (int64_t)idx[a] + axis] < X[3 * (int64_t)idx[b] + axis];
        });
        const size_t half = idx.size() / 2;
        left.clear();
        right.clear();
        for (size_t k = 0; k < order.size(); ++k) (k < half ? left : right).push_back(idx[order[k]]);
    }
    build_node(X, std::move(right), leaf_size, out);
    build_node(X, std::move(left), leaf_size, out);
}

template <class T>
T* upload(const std::vector<T>& v)
{
    if (v.empty()) return nullptr;
    T* d = dalloc<T>(v.size());
    SDFO_CUDA(cudaMemcpy(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return d;
}

} // namespace
} // namespace sdfo

using namespace sdfo;

extern "C" {

int sdfo_contact_pair_create(const sdfo_grid* g, const double* h_quad_x, const double* h_quad_w, int64_t nq,
                             int32_t normalize_weights, double narrow_margin, int32_t leaf_size,
                             sdfo_contact_pair** out)
{
    return guarded([&] {
        SDFO_REQUIRE(out != nullptr, SDFO_ERR_INVALID_ARGUMENT, "out is NULL");
        *out = nullptr;
        SDFO_REQUIRE(nq >= 0 && nq <= 0x7fffffff, SDFO_ERR_INVALID_ARGUMENT, "bad point count");
        SDFO_REQUIRE(nq == 0 || (h_quad_x && h_quad_w), SDFO_ERR_INVALID_ARGUMENT,
                     "quadrature points and weights are required");
        SDFO_REQUIRE(leaf_size >= 1, SDFO_ERR_INVALID_ARGUMENT, "leaf_size must be positive");
        SDFO_REQUIRE(!std::isnan(narrow_margin), SDFO_ERR_INVALID_ARGUMENT, "narrow_margin is NaN");
        std::unique_ptr<sdfo_contact_pair> p(new sdfo_contact_pair());
        p->grid = g;
        p->nq = nq;
        p->narrow_margin = narrow_margin;
        std::vector<double> w(h_quad_w, h_quad_w + nq);
        if (normalize_weights)
        {
            double tot = 0.0; // np.sum (pairwise summation for long arrays; a plain sum here)
            for (double x : w) tot += x;
            if (tot > 1e-30)
                for (double& x : w) x = x / tot;
        }
        std::vector<Leaf> leaves;
        if (nq > 0)
        {
            std::vector<int32_t> all((size_t)nq);
            std::iota(all.begin(), all.end(), 0);
            box_of(h_quad_x, all, p->root);
            build_node(h_quad_x, std::move(all), leaf_size, leaves);
        }
        SDFO_REQUIRE(narrow_margin < 0.0 || (int64_t)leaves.size() <= kMaxCullLeaves, SDFO_ERR_UNSUPPORTED,
                     "too many point-BVH leaves for the culled contact kernel (at most 32768)");
        p->nleaves = (int)leaves.size();
        std::vector<float> px, pw;
        std::vector<int32_t> porig, pleaf;
        std::vector<double> lbox;
        p->h_leaf_start.push_back(0);
        for (size_t l = 0; l < leaves.size(); ++l)
        {
            for (int32_t i : leaves[l].idx)
            {
                for (int a = 0; a < 3; ++a) px.push_back((float)h_quad_x[3 * (int64_t)i + a]);
                pw.push_back((float)w[(size_t)i]);
                porig.push_back(i);
                pleaf.push_back((int32_t)l);
            }
            p->h_leaf_start.push_back((int32_t)porig.size());
            lbox.insert(lbox.end(), leaves[l].box, leaves[l].box + 6);
        }
        p->h_order = porig;
        p->h_leaf_box = lbox;
        if (g == nullptr)
        {
            // the hierarchy alone (export only; evaluation needs a grid)
            *out = p.release();
            return;
        }
        p->px = upload(px);
        p->pw = upload(pw);
        {
            std::vector<double> px64, pw64;
            for (int32_t i : porig)
            {
                for (int a = 0; a < 3; ++a) px64.push_back(h_quad_x[3 * (int64_t)i + a]);
                pw64.push_back(w[(size_t)i]);
            }
            p->px64 = upload(px64);
            p->pw64 = upload(pw64);
            p->ox64 = upload(std::vector<double>(h_quad_x, h_quad_x + 3 * nq));
            p->ow64 = upload(w);
        }
        p->porig = upload(porig);
        p->pleaf = upload(pleaf);
        p->leaf_start = upload(p->h_leaf_start);
        p->leaf_box = upload(lbox);
        *out = p.release();
    });
}

int sdfo_contact_pair_export_bvh(const sdfo_contact_pair* p, int32_t* h_nleaves, int32_t* h_point_order,
                                 int32_t* h_leaf_start, double* h_leaf_box)
{
    return guarded([&] {
        SDFO_REQUIRE(p != nullptr, SDFO_ERR_INVALID_ARGUMENT, "pair is NULL");
        if (h_nleaves) *h_nleaves = p->nleaves;
        if (h_point_order) std::copy(p->h_order.begin(), p->h_order.end(), h_point_order);
        if (h_leaf_start) std::copy(p->h_leaf_start.begin(), p->h_leaf_start.end(), h_leaf_start);
        if (h_leaf_box) std::copy(p->h_leaf_box.begin(), p->h_leaf_box.end(), h_leaf_box);
    });
}

int sdfo_contact_pair_eval(const sdfo_contact_pair* p, int32_t mode, const sdfo_body_state* d_pose_a,
                           int64_t np, const sdfo_body_state* d_body_b, const sdfo_contact_params* h_params,
                           double* d_ft, double* d_jac, sdfo_contact_measure* d_measure, void* stream)
{
    return guarded([&] {
        SDFO_REQUIRE(p != nullptr, SDFO_ERR_INVALID_ARGUMENT, "pair is NULL");
        SDFO_REQUIRE(p->grid != nullptr, SDFO_ERR_INVALID_ARGUMENT, "pair was created without a grid");
        SDFO_REQUIRE(h_params != nullptr, SDFO_ERR_INVALID_ARGUMENT, "contact params are NULL");
        SDFO_REQUIRE(mode == SDFO_TRILINEAR || mode == SDFO_TRICUBIC, SDFO_ERR_UNSUPPORTED,
                     "contact supports Trilinear and Tricubic");
        SDFO_REQUIRE(np >= 0 && np <= 0x7fffffff, SDFO_ERR_INVALID_ARGUMENT, "bad pose count");
        if (np == 0) return;
        SDFO_REQUIRE(d_pose_a && d_body_b, SDFO_ERR_INVALID_ARGUMENT, "poses and body B are required");
        SDFO_REQUIRE(d_ft || d_measure, SDFO_ERR_INVALID_ARGUMENT, "nothing to compute");
        SDFO_REQUIRE(!d_jac || d_ft, SDFO_ERR_INVALID_ARGUMENT, "the Jacobian needs the force output");
        ContactCull c{};
        c.enabled = p->narrow_margin >= 0.0 ? 1 : 0;
        c.nleaves = p->nleaves;
        c.leaf_box = p->leaf_box;
        c.leaf_start = p->leaf_start;
        c.pleaf = p->pleaf;
        c.porig = p->porig;
        for (int a = 0; a < 6; ++a) c.root[a] = p->root[a];
        for (int a = 0; a < 3; ++a)
        {
            c.bmin[a] = p->grid->info.bmin[a];
            c.bmax[a] = p->grid->info.bmax[a];
        }
        c.box_margin = std::max(p->narrow_margin, 0.05);
        c.narrow_margin = p->narrow_margin;
        launch_contact(make_view(p->grid), mode, p->px, p->pw, p->nq, d_pose_a, np, d_body_b, *h_params, d_ft,
                       d_jac, as_stream(stream), &c, d_measure);
    });
}

int sdfo_contact_pair_destroy(sdfo_contact_pair* p)
{
    delete p;
    return SDFO_OK;
}

} // extern "C"
