// Host side of the lag kernel: the per-launch table and the ring's tensor maps.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <limits>
#include <string>
#include <vector>

#include "lag.cuh"

namespace ddm {

// Builds the lag table for one launch. Register frame j (j < nreg) lives in ring slot
// reg[j] (-1: none); entry i pairs register frame j with window position ent_w[i] + j,
// whose ring slot is pos[ent_w[i] + j] (-1: none), into accumulator row ent_acc[i].
// Entries must come with strictly ascending window starts. The windows are merged into the
// sorted list of distinct partner positions (the union); entry i's window is then union
// indices [ub_i, ub_i + nreg), always the tail of the list when the entry is appended
// because windows are contiguous and start in order. The union is cut into groups of
// kLagGroup entries, and each group's valid entries into runs of consecutive ring slots of
// 8, 4, 2 or 1 rows (one tensor-map box each). Returns an empty string on success.
inline std::string build_lag_table(int nreg, const int *reg, const std::vector<int> &ent_acc,
                                   const std::vector<int> &ent_w, const std::vector<int> &pos, int J,
                                   std::vector<int> *table) {
    if (nreg < 1 || nreg > J || J > kLagMaxJ) return "register frame count out of range";
    const int ntau = static_cast<int>(ent_acc.size());
    std::vector<int> ub(ntau), uslot;
    uslot.reserve(pos.size());
    int next = std::numeric_limits<int>::min();  // first position past the union so far
    for (int i = 0; i < ntau; i++) {
        const int w = ent_w[i];
        if (i > 0 && w <= ent_w[i - 1]) return "lag windows out of order";
        if (w < 0 || w + nreg > static_cast<int>(pos.size())) return "lag window outside the position table";
        for (int p = std::max(w, next); p < w + nreg; p++) uslot.push_back(pos[p]);
        next = std::max(next, w + nreg);
        ub[i] = static_cast<int>(uslot.size()) - nreg;
    }
    const int nu = static_cast<int>(uslot.size());
    bool regs_ok = nreg == J;
    for (int j = 0; j < nreg; j++) regs_ok = regs_ok && reg[j] >= 0;
    std::vector<int> full(ntau);
    for (int i = 0; i < ntau; i++) {
        bool f = regs_ok;
        for (int j = 0; j < nreg && f; j++) f = uslot[ub[i] + j] >= 0;
        full[i] = f ? 1 : 0;
    }
    // runs of kLagFuse full entries whose windows start one union entry apart
    for (int i = 0; i + kLagFuse <= ntau;) {
        bool run = true;
        for (int r = 0; r < kLagFuse && run; r++) run = full[i + r] && ub[i + r] == ub[i] + r;
        if (run) {
            full[i] |= kLagRunFlag;
            i += kLagFuse;
        } else {
            i++;
        }
    }
    const int ngroups = (nu + kLagGroup - 1) / kLagGroup;
    std::vector<int> gptr(ngroups + 1, 0), runs;
    for (int g = 0; g < ngroups; g++) {
        const int u0 = g * kLagGroup, u1 = std::min(nu, u0 + kLagGroup);
        for (int u = u0; u < u1;) {
            if (uslot[u] < 0) {
                u++;
                continue;
            }
            int len = 1;  // consecutive ring slots
            while (u + len < u1 && uslot[u + len] == uslot[u] + len) len++;
            while (len > 0) {  // split into boxes of 8, 4, 2, 1 rows
                int lg = 3;
                while ((1 << lg) > len) lg--;
                if (uslot[u] > 0xFFFFF) return "ring slot index too large for a lag run";
                runs.push_back(lag_run(u - u0, uslot[u], lg));
                u += 1 << lg;
                len -= 1 << lg;
            }
        }
        gptr[g + 1] = static_cast<int>(runs.size());
    }
    const int nruns = static_cast<int>(runs.size());
    table->assign(lag_table_ints(ntau, nu, ngroups, nruns), 0);
    int *t = table->data();
    t[kTabNreg] = nreg;
    t[kTabNtau] = ntau;
    t[kTabNunion] = nu;
    t[kTabNgroups] = ngroups;
    t[kTabNruns] = nruns;
    for (int j = 0; j < kLagMaxJ; j++) t[kTabReg + j] = j < nreg ? reg[j] : -1;
    int *p = t + kTabEntries;
    p = std::copy(ent_acc.begin(), ent_acc.end(), p);
    p = std::copy(ub.begin(), ub.end(), p);
    p = std::copy(full.begin(), full.end(), p);
    p = std::copy(uslot.begin(), uslot.end(), p);
    p = std::copy(gptr.begin(), gptr.end(), p);
    std::copy(runs.begin(), runs.end(), p);
    return std::string();
}

// Upper bound of the table size for ntau entries over npos window positions.
inline int lag_table_capacity(int ntau, int npos) {
    const int nu = npos, ngroups = (nu + kLagGroup - 1) / kLagGroup;
    return lag_table_ints(ntau, nu, ngroups, nu);
}

// Smallest instantiated register-frame count >= nreg (0 if none).
inline int lag_pick_j(int nreg) {
    for (int J : kLagJs)
        if (J >= nreg) return J;
    return 0;
}

// Tensor maps of a ring float2[slots][E] for boxes of 128 or 64 elements (the element blocks
// of the one- and two-lane kernels) x 1, 2, 4, 8 slots.
inline std::string make_lag_maps(const void *ring, long long E, int slots, LagMaps *maps) {
    // looked up once, by a thread-safe static initialiser (engines on several threads and
    // the static entry point all come through here)
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) return "cuTensorMapEncodeTiled is not available from the driver";
    if (reinterpret_cast<uintptr_t>(ring) % 16 != 0) return "the ring must start on a 16-byte boundary";
    if ((E * 8) % 16 != 0) return "frame size must be a multiple of 16 bytes for the ring tensor maps";
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(E), static_cast<cuuint64_t>(slots)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(E) * 8};
    const cuuint32_t estr[2] = {1, 1};
    const int widths[2] = {lag_cta_elems(1), lag_cta_elems(kLagMaxJ)};
    for (int w = 0; w < 2; w++) {
        for (int k = 0; k < kLagRunKinds; k++) {
            const cuuint32_t box[2] = {static_cast<cuuint32_t>(widths[w]), 1u << k};
            CUresult r = encode(&maps->box[w][k], CU_TENSOR_MAP_DATA_TYPE_INT64, 2, const_cast<void *>(ring), dims,
                                strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS)
                return "cuTensorMapEncodeTiled failed with code " + std::to_string(static_cast<int>(r));
        }
    }
    return std::string();
}

}  // namespace ddm
