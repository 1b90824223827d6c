// Host-side system assembly: the reference's input builders in C++.
//
//   gcmc_cavity_grid   -- GCMCDataset.get_grid   (gcmc/python/dataset.py:21-139)
//   gcmc_fix_groups    -- GCMCDataset.set_fixCut (gcmc/python/dataset.py:175-188)
//   gcmc_group_centres -- the residue centres of update_data (gcmc/python/dataset.py:248-300)
//   gcmc_fill_layout   -- update_data's residue / atom arrays (gcmc/python/dataset.py:190-373)
//
// The arithmetic follows the reference's Python/numpy (under its numpy<2
// dependency) so that the outputs are identical: float64 geometry, centres as
// float32 running sums of float64 additions divided in float64, voxel indices
// by truncation and Python's non-negative modulo.  Differences are deliberate
// and few: empty voxels come out in lexicographic (x, y, z) order instead of
// Python set order, and unused slots are zero-filled.
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/gcmc_b200.h"

namespace {

constexpr int kMaxSitesAbi = 20;  // AtomArray.atoms[20]

inline int64_t pymod(int64_t a, int64_t n) {
    const int64_t r = a % n;
    return r < 0 ? r + n : r;
}

// float32 running sum of float64 additions, then a float64 division (numpy<2
// semantics of `float32 += float64` followed by `/ n`).
inline void centre_of(const double* xyz, int64_t start, int32_t count, float out[3]) {
    float acc[3] = {0.0f, 0.0f, 0.0f};
    for (int32_t j = 0; j < count; ++j)
        for (int c = 0; c < 3; ++c) acc[c] = (float)((double)acc[c] + xyz[(start + j) * 3 + c]);
    const double n = count > 0 ? (double)count : 1.0;
    for (int c = 0; c < 3; ++c) out[c] = (float)((double)acc[c] / n);
}

// The voxel lattice of get_grid and which voxels hold an atom (occ empty
// without cavity bias: every voxel of a 1 A grid is a base point).
struct CavityVoxels {
    double start[3], dx, factor;
    int64_t nv[3], nempty;
    std::vector<uint8_t> occ;
};

int cavity_voxels(int32_t n, const double* xyz, const double* cryst, double grid_dx, int32_t cavity_bias,
                  CavityVoxels* cv) {
    if (n < 1 || !xyz || !cryst) return GCMC_ERR_ARG;
    double lo[3], hi[3];
    for (int c = 0; c < 3; ++c) lo[c] = hi[c] = xyz[c];
    for (int32_t a = 1; a < n; ++a)
        for (int c = 0; c < 3; ++c) {
            lo[c] = std::fmin(lo[c], xyz[3 * a + c]);
            hi[c] = std::fmax(hi[c], xyz[3 * a + c]);
        }
    cv->dx = cavity_bias ? grid_dx : 1.0;
    for (int c = 0; c < 3; ++c) {
        const double centre = (lo[c] + hi[c]) / 2.0;
        cv->start[c] = centre - cryst[c] / 2.0;
        const double end = centre + cryst[c] / 2.0;
        cv->nv[c] = (int64_t)((end - cv->start[c]) / cv->dx);
        if (cv->nv[c] < 1) return GCMC_ERR_ARG;
    }
    const int64_t total = cv->nv[0] * cv->nv[1] * cv->nv[2];
    cv->occ.clear();
    int64_t nocc = 0;
    if (cavity_bias) {
        cv->occ.assign((size_t)total, 0);
        for (int32_t a = 0; a < n; ++a) {
            int64_t v[3];
            for (int c = 0; c < 3; ++c)
                v[c] = pymod((int64_t)std::trunc((xyz[3 * a + c] - cv->start[c]) / cv->dx), cv->nv[c]);
            uint8_t& o = cv->occ[(size_t)((v[0] * cv->nv[1] + v[1]) * cv->nv[2] + v[2])];
            nocc += !o;
            o = 1;
        }
    }
    cv->nempty = total - nocc;
    cv->factor = cavity_bias ? (double)cv->nempty / (double)total : 1.0;
    return GCMC_OK;
}

}  // namespace

extern "C" {

int gcmc_cavity_grid(int32_t n, const double* xyz, const double* cryst, double grid_dx, int32_t cavity_bias,
                     double* start, float* pts, int64_t cap, int64_t* npts, double* factor) {
    if (!start || !npts || !factor) return GCMC_ERR_ARG;
    CavityVoxels cv;
    const int st = cavity_voxels(n, xyz, cryst, grid_dx, cavity_bias, &cv);
    if (st != GCMC_OK) return st;
    for (int c = 0; c < 3; ++c) start[c] = cv.start[c];
    *npts = cv.nempty;
    *factor = cv.factor;
    if (cavity_bias && cv.factor < 0.05) return GCMC_ERR_ARG;  // the reference exits here (dataset.py:95-97)
    if (!pts) return GCMC_OK;
    if (cap < cv.nempty) return GCMC_ERR_LIMIT;
    int64_t k = 0;
    for (int64_t x = 0; x < cv.nv[0]; ++x)
        for (int64_t y = 0; y < cv.nv[1]; ++y)
            for (int64_t z = 0; z < cv.nv[2]; ++z) {
                if (!cv.occ.empty() && cv.occ[(size_t)((x * cv.nv[1] + y) * cv.nv[2] + z)]) continue;
                pts[3 * k] = (float)((double)x * cv.dx + cv.start[0]);
                pts[3 * k + 1] = (float)((double)y * cv.dx + cv.start[1]);
                pts[3 * k + 2] = (float)((double)z * cv.dx + cv.start[2]);
                ++k;
            }
    return GCMC_OK;
}

int gcmc_cavity_bits(int32_t n, const double* xyz, const double* cryst, double grid_dx, int32_t cavity_bias,
                     gcmc_grid_bits* hdr, uint32_t* words, int64_t cap_words, int64_t* nwords, int64_t* npts) {
    if (!hdr || !nwords || !npts) return GCMC_ERR_ARG;
    CavityVoxels cv;
    const int st = cavity_voxels(n, xyz, cryst, grid_dx, cavity_bias, &cv);
    if (st != GCMC_OK) return st;
    for (int c = 0; c < 3; ++c) {
        if (cv.nv[c] > INT32_MAX) return GCMC_ERR_LIMIT;
        hdr->start[c] = cv.start[c];
        hdr->n[c] = (int32_t)cv.nv[c];
    }
    hdr->dx = cv.dx;
    hdr->pad = 0;
    const int64_t total = cv.nv[0] * cv.nv[1] * cv.nv[2];
    *nwords = (total + 31) / 32;
    *npts = cv.nempty;
    if (cavity_bias && cv.factor < 0.05) return GCMC_ERR_ARG;
    if (!words) return GCMC_OK;
    if (cap_words < *nwords) return GCMC_ERR_LIMIT;
    std::memset(words, 0, sizeof(uint32_t) * (size_t)*nwords);
    for (int64_t v = 0; v < total; ++v)
        if (cv.occ.empty() || !cv.occ[(size_t)v]) words[v >> 5] |= 1u << (v & 31);
    return GCMC_OK;
}

int32_t gcmc_fix_groups(int32_t n, const double* xyz, double fix_cutoff, int32_t* group) {
    if (n < 0 || (n > 0 && (!xyz || !group))) return -1;
    double x0 = INFINITY, y0 = INFINITY, z0 = INFINITY;
    int32_t g = -1;
    for (int32_t i = 0; i < n; ++i) {
        const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        if (std::sqrt((x - x0) * (x - x0) + (y - y0) * (y - y0) + (z - z0) * (z - z0)) > fix_cutoff) {
            ++g;
            x0 = x; y0 = y; z0 = z;
        }
        group[i] = g;
    }
    return g + 1;
}

int gcmc_group_centres(int32_t ngroups, const double* xyz, const int64_t* starts, const int32_t* counts,
                       float* out) {
    if (ngroups < 0 || (ngroups > 0 && (!xyz || !starts || !counts || !out))) return GCMC_ERR_ARG;
    for (int32_t g = 0; g < ngroups; ++g) centre_of(xyz, starts[g], counts[g], out + 3 * g);
    return GCMC_OK;
}

int gcmc_fill_layout(int32_t nfix, const double* fixed_xyz, const double* fixed_q, const int32_t* fixed_type,
                     const int32_t* fixed_group, int32_t nfrag, const int32_t* max_num, const int32_t* num_atoms,
                     const float* tpl_q, const int32_t* tpl_type, const int32_t* n_initial,
                     const double* initial_xyz, int32_t total_res, int64_t total_atoms, residue* res, Atom* atoms,
                     int32_t* start_res) {
    if (nfix < 0 || nfrag < 0 || !res || !atoms || !start_res) return GCMC_ERR_ARG;
    std::memset(res, 0, sizeof(residue) * (size_t)total_res);
    std::memset(atoms, 0, sizeof(Atom) * (size_t)total_atoms);
    // fixed atoms and their groups (contiguous runs of equal group id)
    int32_t seq = 0;
    int64_t a = 0;
    while (a < nfix) {
        int64_t b = a;
        while (b < nfix && fixed_group[b] == fixed_group[a]) ++b;
        if (seq >= total_res) return GCMC_ERR_LIMIT;
        res[seq].atomStart = (int32_t)a;
        res[seq].atomNum = (int32_t)(b - a);
        centre_of(fixed_xyz, a, (int32_t)(b - a), res[seq].position);
        ++seq;
        a = b;
    }
    if (nfix > total_atoms) return GCMC_ERR_LIMIT;
    for (int64_t i = 0; i < nfix; ++i) {
        for (int c = 0; c < 3; ++c) atoms[i].position[c] = (float)fixed_xyz[3 * i + c];
        atoms[i].charge = (float)fixed_q[i];
        atoms[i].type = fixed_type[i];
    }
    // fragment slots: maxNum per type, the first n_initial filled
    int64_t next = nfix, tq = 0, ix = 0;
    for (int32_t f = 0; f < nfrag; ++f) {
        start_res[f] = seq;
        const int32_t na = num_atoms[f];
        for (int32_t j = 0; j < max_num[f]; ++j) {
            if (seq >= total_res || next + na > total_atoms) return GCMC_ERR_LIMIT;
            res[seq].atomNum = na;
            res[seq].atomStart = (int32_t)next;
            if (j < n_initial[f]) {
                for (int32_t s = 0; s < na; ++s) {
                    for (int c = 0; c < 3; ++c) atoms[next + s].position[c] = (float)initial_xyz[(ix + s) * 3 + c];
                    atoms[next + s].charge = tpl_q[tq + s];
                    atoms[next + s].type = tpl_type[tq + s];
                }
                centre_of(initial_xyz, ix, na, res[seq].position);
                ix += na;
            }
            next += na;
            ++seq;
        }
        tq += na;
    }
    return GCMC_OK;
}

}  // extern "C"

extern "C" {

// get_data's fragment records (gcmc/python/dataset.py:393-408): one ATOM line
// per atom of every occupied slot, in type and slot order, serials and residue
// numbers continuing from serial0 / resnum0 and wrapping at 99999 / 9999.
// atom_names: per type 20 names of 4 chars (not NUL-terminated).  Returns the
// number of bytes written, or (out == NULL or cap too small) the number needed.
int64_t gcmc_pdb_fragment_lines(int32_t nfrag, const AtomArray* fragmentInfo, const residue* residueInfo,
                                const Atom* atomInfo, const char* atom_names, int64_t serial0, int64_t resnum0,
                                char* out, int64_t cap) {
    if (nfrag < 0 || !fragmentInfo || !residueInfo || !atomInfo || !atom_names) return -1;
    int64_t need = 0;
    for (int32_t i = 0; i < nfrag; ++i) need += (int64_t)fragmentInfo[i].totalNum * fragmentInfo[i].num_atoms;
    // a record is 66 bytes while every coordinate fits %8.3f; 96 bounds any line
    if (!out || cap < need * 96) return need * 96;
    int64_t pos = 0, serial = serial0, resnum = resnum0;
    char buf[160];
    for (int32_t i = 0; i < nfrag; ++i) {
        const AtomArray& F = fragmentInfo[i];
        for (int32_t j = 0; j < F.totalNum; ++j) {
            const residue& r = residueInfo[F.startRes + j];
            for (int32_t k = 0; k < r.atomNum; ++k) {
                const Atom& a = atomInfo[r.atomStart + k];
                const char* nm = atom_names + ((size_t)i * kMaxSitesAbi + k) * 4;
                const int len = std::snprintf(buf, sizeof(buf), "ATOM  %5lld  %-4.4s%-4.4s %4lld    %8.3f%8.3f%8.3f  1.00  0.00\n",
                                              (long long)((serial - 1) % 99999 + 1), nm, F.name,
                                              (long long)((resnum - 1) % 9999 + 1), (double)a.position[0],
                                              (double)a.position[1], (double)a.position[2]);
                if (len <= 0 || pos + len > cap) return -1;
                std::memcpy(out + pos, buf, (size_t)len);
                pos += len;
                ++serial;
            }
            ++resnum;
        }
    }
    return pos;
}

}  // extern "C"
