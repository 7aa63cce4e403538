// mrhs.cu — task tables of the multi-RHS solve (k_sptrsv_mrhs).
//
// Built on the host from the plan's level layout (positions in level order,
// ptr[] giving each position's off-diagonal range) and the rows' levels:
// per level, every long row (more off-diagonals than one wait round of a
// lane covers) is cut into pieces of about P = 2 rounds of the warp's
// E = 32/kp element slots, and the short rows are packed E to a group.  A
// level's pieces come first, so the longest work of a level starts first on
// the persistent warps, which take tasks round-robin in table order.
#include <algorithm>
#include <vector>

#include "internal.h"
#include "plan.h"
#include "solve_kernels.cuh"

namespace sptrsv {

namespace {
constexpr int kMrhsU = 15;       // at most this many entries per lane of a group row
constexpr int kPieceRounds = 1;  // wait rounds per piece of a long row
static_assert(kMrhsU <= 15, "group row lengths are packed in 4 bits");
}

void mrhs_free(MrhsTable& t)
{
    cudaFree(t.tasks);
    cudaFree(t.pbuf);
    cudaFree(t.pcnt);
    t = MrhsTable();
}

int build_mrhs_tasks(sptrsv_plan_s* p, int kp, int U)
{
    int j = 0;
    while ((1 << j) < kp) j++;
    MrhsTable& t = p->mrhs[j];
    if (t.tasks && t.U == U) return 0;
    if (t.tasks) mrhs_free(t);
    const int n = p->n, E = 32 / kp;
    const int short_max = std::min(U, kMrhsU);  // a GROUP row is one wait round of its lanes
    const int piece = kPieceRounds * E * U;  // a PIECE is kPieceRounds wait rounds of the warp
    std::vector<int> ptr(n + 1), rowid(n), lev(n);
    SPT_CUDA(cudaMemcpy(ptr.data(), p->lev.ptr, sizeof(int) * (size_t)(n + 1), cudaMemcpyDeviceToHost));
    SPT_CUDA(cudaMemcpy(rowid.data(), p->lev.rowid, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
    SPT_CUDA(cudaMemcpy(lev.data(), p->levels, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
    std::vector<MrhsTask> tasks, groups;
    tasks.reserve((size_t)n / 2 + 16);
    int npslots = 0, nsplit = 0;
    for (int a = 0; a < n;) {
        const int L = lev[rowid[a]];
        int bnd = a;
        while (bnd < n && lev[rowid[bnd]] == L) bnd++;
        groups.clear();
        for (int k = a; k < bnd;) {
            const int len = ptr[k + 1] - ptr[k];
            if (len > short_max) {
                const int np = (len + piece - 1) / piece, chunk = (len + np - 1) / np;
                const int ps = npslots, cs = nsplit;
                for (int q = 0; q < np; q++) {
                    MrhsTask x{};
                    x.pos = k;
                    x.cnt = -np;
                    x.e0 = ptr[k] + q * chunk;
                    x.e1 = std::min(ptr[k + 1], x.e0 + chunk);
                    x.pslot = ps + q;
                    x.cslot = cs;
                    x.piece = q;
                    tasks.push_back(x);
                }
                if (np > 1) {
                    npslots += np;
                    nsplit++;
                }
                k++;
                continue;
            }
            int c = 1;
            while (c < E && k + c < bnd && ptr[k + c + 1] - ptr[k + c] <= short_max) c++;
            MrhsTask g{};
            g.pos = k;
            g.cnt = c;
            g.e0 = ptr[k];  // the group's entries are contiguous from here
            unsigned long long lens = 0;
            for (int i = 0; i < c; i++) lens |= (unsigned long long)(ptr[k + i + 1] - ptr[k + i]) << (4 * i);
            g.e1 = (int)(unsigned)(lens & 0xffffffffu);
            g.pslot = (int)(unsigned)(lens >> 32);
            groups.push_back(g);
            k += c;
        }
        tasks.insert(tasks.end(), groups.begin(), groups.end());
        a = bnd;
    }
    MrhsTable nt;
    nt.ntasks = (int)tasks.size();
    nt.npslots = npslots;
    nt.nsplit = nsplit;
    nt.U = U;
    auto fail = [&](cudaError_t e) {
        mrhs_free(nt);
        return cuda_fail(e, "build_mrhs_tasks");
    };
    cudaError_t e = dalloc(&nt.tasks, (long long)nt.ntasks * 8);
    if (e == cudaSuccess && nt.ntasks)
        e = cudaMemcpy(nt.tasks, tasks.data(), sizeof(MrhsTask) * tasks.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&nt.pbuf, sizeof(double) * (size_t)std::max(1, npslots) * kp);
    if (e == cudaSuccess) e = dalloc(&nt.pcnt, std::max(1, nsplit));
    if (e != cudaSuccess) return fail(e);
    t = nt;
    return 0;
}

}  // namespace sptrsv
