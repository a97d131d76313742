// Host-side mesh set-up of libvbd_b200: greedy vertex colouring, lumped masses, rest-shape
// inverses.  Pure integer / FP32 host work, run once per mesh; no GPU needed.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "vbd_b200.h"
#include "vbd_internal.h"

namespace vbd {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

void clear_error() { g_last_error.clear(); }

const char* last_error() { return g_last_error.c_str(); }

int check_tets(int32_t num_verts, int32_t num_tets, const int32_t* tets) {
    if (num_verts < 0 || num_tets < 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "negative mesh size");
    if (num_tets > 0 && !tets) VBD_FAIL(VBD_ERR_INVALID_ARG, "tets is null");
    for (int64_t t = 0; t < num_tets; ++t) {
        const int32_t* q = tets + 4 * t;
        for (int a = 0; a < 4; ++a) {
            if (q[a] < 0 || q[a] >= num_verts)
                VBD_FAIL(VBD_ERR_INVALID_ARG, "tet %lld holds vertex id %d outside [0, %d)", (long long)t, q[a],
                         num_verts);
            for (int b = 0; b < a; ++b)
                if (q[a] == q[b])
                    VBD_FAIL(VBD_ERR_INVALID_ARG, "tet %lld repeats vertex id %d", (long long)t, q[a]);
        }
    }
    return VBD_OK;
}

void build_vertex_tets(int32_t num_verts, int32_t num_tets, const int32_t* tets, int32_t* offsets,
                       int32_t* tet_ids) {
    std::fill(offsets, offsets + num_verts + 1, 0);
    for (int64_t k = 0; k < 4LL * num_tets; ++k) offsets[tets[k] + 1]++;
    for (int32_t i = 0; i < num_verts; ++i) offsets[i + 1] += offsets[i];
    std::vector<int32_t> fill(offsets, offsets + num_verts);
    // Tets visited in ascending id, so each vertex's list comes out ascending.
    for (int32_t t = 0; t < num_tets; ++t)
        for (int a = 0; a < 4; ++a) tet_ids[fill[tets[4 * t + a]]++] = t;
}

// Largest relative error, over every tet and local vertex n, of det M as the factored record
// layouts obtain it in FP32, against det M in FP64 of the same FP32 rows.  M is the 3x3 matrix of
// the other three rows q_k of Q = Ps Dm^-1 and q_n = -(q_a + q_b + q_c).  Layout 3 stores det M =
// M_0 . cof(M)_0; layout 4 derives it as s.w / |q_n|^2 with s = M q_n, w = cof(M) q_n and |q_n|^2 =
// -(s_0 + s_1 + s_2), which cancels when |q_n| is small next to the other rows (anisotropic or
// sliver tets).  The FP32 steps follow k_pack_factored and decode_fact.
void factored_detm_error(int32_t num_tets, const float* dm_inv, double* err3, double* err4, double* frac4) {
    double e3 = 0.0, e4 = 0.0;
    long long counted = 0, over = 0;
    for (int64_t t = 0; t < num_tets; ++t) {
        const float* d = dm_inv + 9 * t;
        float Q[4][3];
        for (int c = 0; c < 3; ++c) {
            Q[0][c] = -d[c] - d[3 + c] - d[6 + c];
            for (int k = 1; k < 4; ++k) Q[k][c] = d[3 * (k - 1) + c];
        }
        for (int n = 0; n < 4; ++n) {
            float M[3][3];
            int m = 0;
            for (int k = 0; k < 4; ++k) {
                if (k == n) continue;
                for (int c = 0; c < 3; ++c) M[m][c] = Q[k][c];
                ++m;
            }
            const float q[3] = {-(M[0][0] + M[1][0] + M[2][0]), -(M[0][1] + M[1][1] + M[2][1]),
                                -(M[0][2] + M[1][2] + M[2][2])};
            float cof[3][3];
            for (int i = 0; i < 3; ++i) {
                const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
                for (int c = 0; c < 3; ++c) {
                    const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
                    cof[i][c] = M[i1][c1] * M[i2][c2] - M[i1][c2] * M[i2][c1];
                }
            }
            float sv[3], wv[3];
            for (int i = 0; i < 3; ++i) {
                sv[i] = M[i][0] * q[0] + M[i][1] * q[1] + M[i][2] * q[2];
                wv[i] = cof[i][0] * q[0] + cof[i][1] * q[1] + cof[i][2] * q[2];
            }
            const float det3 = M[0][0] * cof[0][0] + M[0][1] * cof[0][1] + M[0][2] * cof[0][2];
            const float qq = -(sv[0] + sv[1] + sv[2]);
            const float sw = std::fma(sv[2], wv[2], std::fma(sv[1], wv[1], sv[0] * wv[0]));
            const float det4 = sw / qq;
            double Md[3][3];
            for (int i = 0; i < 3; ++i)
                for (int c = 0; c < 3; ++c) Md[i][c] = M[i][c];
            const double exact = Md[0][0] * (Md[1][1] * Md[2][2] - Md[1][2] * Md[2][1]) -
                                 Md[0][1] * (Md[1][0] * Md[2][2] - Md[1][2] * Md[2][0]) +
                                 Md[0][2] * (Md[1][0] * Md[2][1] - Md[1][1] * Md[2][0]);
            if (exact == 0.0 || !std::isfinite(exact)) {
                e3 = e4 = INFINITY;
                continue;
            }
            const double r3 = std::fabs((double)det3 / exact - 1.0), r4 = std::fabs((double)det4 / exact - 1.0);
            e3 = std::isfinite(r3) ? std::max(e3, r3) : INFINITY;
            e4 = std::isfinite(r4) ? std::max(e4, r4) : INFINITY;
            // Does layout 4 lose accuracy here: is its error above the tolerance and above a few
            // times the stored det M's own error (the conditioning of Dm^-1)?  Tets that are
            // degenerate in FP32 (the stored det M already off by more than kFactoredDegenerate)
            // give no usable element in any FP32 form and are left out.
            if (std::isfinite(r3) && r3 > kFactoredDegenerate) continue;
            ++counted;
            if (!(r4 <= std::max(kFactoredDetmTol, kFactoredDetmRatio * r3))) ++over;
        }
    }
    if (err3) *err3 = e3;
    if (err4) *err4 = e4;
    if (frac4) *frac4 = counted ? (double)over / (double)counted : 0.0;
}

}  // namespace vbd

extern "C" {

int vbd_factored_record_error(int32_t num_tets, const float* dm_inv, double* err_layout3, double* err_layout4,
                              double* layout4_loss_fraction) {
    vbd::clear_error();
    if (num_tets < 0 || (num_tets > 0 && !dm_inv)) VBD_FAIL(VBD_ERR_INVALID_ARG, "need dm_inv[9 * num_tets]");
    vbd::factored_detm_error(num_tets, dm_inv, err_layout3, err_layout4, layout4_loss_fraction);
    return VBD_OK;
}

int vbd_version(void) { return 100; }

const char* vbd_last_error(void) { return vbd::last_error(); }

int vbd_color_vertices(int32_t num_verts, int32_t num_tets, const int32_t* tets, int32_t* colour_of,
                       int32_t* num_colours, int32_t max_colours, int32_t* group_offsets,
                       int32_t* group_vertices) {
    vbd::clear_error();
    if (!colour_of || !num_colours) VBD_FAIL(VBD_ERR_INVALID_ARG, "colour_of / num_colours is null");
    if (int rc = vbd::check_tets(num_verts, num_tets, tets)) return rc;
    std::vector<int32_t> off(num_verts + 1), vt(4LL * num_tets);
    vbd::build_vertex_tets(num_verts, num_tets, tets, off.data(), vt.data());
    // Greedy pass in vertex-id order.  A neighbour's colour counts only once it is assigned,
    // i.e. for neighbours with a smaller id; used colours are marked with the current vertex's
    // stamp so the scratch array never needs clearing.
    std::vector<int32_t> stamp(64, -1);
    int32_t ncol = 0;
    for (int32_t v = 0; v < num_verts; ++v) colour_of[v] = -1;
    for (int32_t v = 0; v < num_verts; ++v) {
        for (int32_t k = off[v]; k < off[v + 1]; ++k) {
            const int32_t* q = tets + 4LL * vt[k];
            for (int a = 0; a < 4; ++a) {
                int32_t nb = q[a];
                if (nb == v) continue;
                int32_t c = colour_of[nb];
                if (c >= 0) stamp[c] = v;
            }
        }
        int32_t c = 0;
        while (c < (int32_t)stamp.size() && stamp[c] == v) ++c;
        if (c + 1 >= (int32_t)stamp.size()) stamp.resize(2 * stamp.size() + 2, -1);
        colour_of[v] = c;
        if (c + 1 > ncol) ncol = c + 1;
    }
    *num_colours = ncol;
    if (group_offsets || group_vertices) {
        if (!group_offsets || !group_vertices)
            VBD_FAIL(VBD_ERR_INVALID_ARG, "group_offsets and group_vertices must both be given");
        if (max_colours < ncol)
            VBD_FAIL(VBD_ERR_INVALID_ARG, "mesh needs %d colours, capacity is %d", ncol, max_colours);
        std::fill(group_offsets, group_offsets + ncol + 1, 0);
        for (int32_t v = 0; v < num_verts; ++v) group_offsets[colour_of[v] + 1]++;
        for (int32_t c = 0; c < ncol; ++c) group_offsets[c + 1] += group_offsets[c];
        std::vector<int32_t> fill(group_offsets, group_offsets + ncol);
        for (int32_t v = 0; v < num_verts; ++v) group_vertices[fill[colour_of[v]]++] = v;
    }
    return VBD_OK;
}

int vbd_mesh_mass(int32_t num_verts, int32_t num_tets, const float* rest_xyz, const int32_t* tets,
                  float density, float* vertex_mass, float* tet_rest_vol) {
    vbd::clear_error();
    if (!rest_xyz && num_verts > 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "rest_xyz is null");
    if (int rc = vbd::check_tets(num_verts, num_tets, tets)) return rc;
    if (vertex_mass)
        for (int32_t i = 0; i < num_verts; ++i) vertex_mass[i] = 0.0f;
    for (int32_t t = 0; t < num_tets; ++t) {
        const int32_t* q = tets + 4LL * t;
        const float* o = rest_xyz + 3LL * q[0];
        float e[3][3];
        for (int k = 0; k < 3; ++k)
            for (int r = 0; r < 3; ++r) e[k][r] = rest_xyz[3LL * q[k + 1] + r] - o[r];
        // e0 . (e1 x e2), accumulated left to right
        float c0 = e[1][1] * e[2][2] - e[1][2] * e[2][1];
        float c1 = e[1][2] * e[2][0] - e[1][0] * e[2][2];
        float c2 = e[1][0] * e[2][1] - e[1][1] * e[2][0];
        float d = e[0][0] * c0;
        d += e[0][1] * c1;
        d += e[0][2] * c2;
        float vol = std::fabs(d) / 6.0f;
        if (tet_rest_vol) tet_rest_vol[t] = vol;
        if (vertex_mass) {
            float share = (vol * density) / 4.0f;
            for (int a = 0; a < 4; ++a) vertex_mass[q[a]] += share;
        }
    }
    return VBD_OK;
}

int vbd_precompute_tets(int32_t num_verts, int32_t num_tets, const float* rest_xyz, const int32_t* tets,
                        float* dm_inv, float* rest_vol) {
    vbd::clear_error();
    if (!rest_xyz && num_verts > 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "rest_xyz is null");
    if (int rc = vbd::check_tets(num_verts, num_tets, tets)) return rc;
    for (int32_t t = 0; t < num_tets; ++t) {
        const int32_t* q = tets + 4LL * t;
        float D[3][3];  // columns x1-x0, x2-x0, x3-x0
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) D[r][c] = rest_xyz[3LL * q[c + 1] + r] - rest_xyz[3LL * q[0] + r];
        if (dm_inv) {
            // adjugate / determinant; cofactor (i,j) from the cyclic successors of i and j
            auto cof = [&](int i, int j) {
                int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                return D[i1][j1] * D[i2][j2] - D[i1][j2] * D[i2][j1];
            };
            float k0 = cof(0, 0), k1 = cof(1, 0), k2 = cof(2, 0);
            float det = k0 * D[0][0];
            det += k1 * D[1][0];
            det += k2 * D[2][0];
            float inv = 1.0f / det;
            float* o = dm_inv + 9LL * t;
            o[0] = k0 * inv;
            o[1] = k1 * inv;
            o[2] = k2 * inv;
            for (int r = 1; r < 3; ++r)
                for (int c = 0; c < 3; ++c) o[3 * r + c] = cof(c, r) * inv;
        }
        if (rest_vol) {
            // |d3 . (d1 x d2)| / 6 with d_k the columns
            float x1 = D[1][0] * D[2][1] - D[2][0] * D[1][1];
            float x2 = D[2][0] * D[0][1] - D[0][0] * D[2][1];
            float x3 = D[0][0] * D[1][1] - D[1][0] * D[0][1];
            float d = D[0][2] * x1;
            d += D[1][2] * x2;
            d += D[2][2] * x3;
            rest_vol[t] = std::fabs(d) / 6.0f;
        }
    }
    return VBD_OK;
}

}  // extern "C"
