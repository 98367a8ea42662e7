// Batch contour kernel (FP64): the propagator chains of many SCFT instances in ONE
// persistent cooperative launch.
//
// Each chain (forward q or backward q+ of one instance, src/crysSCFT_sample.cpp:483-491)
// runs on a team of T CTAs with the alternating-layout schedule of contour_alt_kernel
// (plane phase [A_z A_y] D store D [A_y], slab phase [A_z A_x] D store D [A_x], one
// exchange per step through the chain's exchange buffers).  Where contour_alt_kernel gives
// every unit (x-plane or y-slab) its own CTA, a team CTA owns P = n / T units (rank,
// rank + T, ...) and runs them one after the other in every phase, so a chain occupies T
// SMs instead of n and one exchange latency per step is shared by P units of work.
// Synchronisation is per phase and CTA pair: a CTA waits once per phase for one flag of
// every producer CTA of its team, and releases its own flags once, after its last unit;
// while a unit's last axis operation runs, the next unit's tile is fetched into the work
// tile the unit no longer reads.  Every unit does exactly the arithmetic of
// contour_alt_kernel (same tile operations and epilogues, in the same order), so the
// results are bit-identical to the per-instance kernel.
//
// Scheduling: the host (team_schedule in scft.cu) gives every CTA an ordered task list
// (chain, rank, team size).  CTAs are grouped in columns of one team size; every CTA of a
// column runs the same chains in the same order, so a team never waits for a member busy
// with another task and the launch cannot deadlock.  Every wait is bounded; a CTA that
// gives up sets the batch's abort word, which every other wait polls, drains its own bulk
// copies and leaves.
#pragma once

namespace crysscft {

// One chain of one instance as the batch kernel sees it (device memory, 64-byte aligned).
struct TeamChain {
    alignas(64) CUtensorMap tm_q[2];     // contour store in 8-column panels: plane [0] / slab [1] view
    alignas(64) CUtensorMap tm_w[2][2];  // Boltzmann factors exp(-w ds/2) [block A, B][view]
    double* q;                           // contour store (slot0 is the chain's input)
    double* xbuf;                        // 2 x space_size_phy: plane-phase then slab-phase exchange buffer
    const double* ops;                   // packed operators (two-level block for form 0)
    unsigned* flags;                     // [layout][consumer CTA][producer CTA], room for 2 n^2; zeroed before the launch
    unsigned* error;                     // the instance's error word (same bits as contour_alt_kernel)
    long long slot0;                     // first input slot
    long long NsA;                       // segments < NsA use block A's factors
    int dir;                             // +1 forward, -1 backward
    int U;                               // contour steps
    int n;                               // cubic physical grid side
    int form;                            // tile form (TeamForm)
};

// (chain, rank in team, team size) of one CTA's task
struct TeamTask {
    int chain;
    int rank;
    int size;
    int pad;
};

struct BatchContourArgs {
    const TeamChain* chains;
    const TeamTask* tasks;   // CTA b runs tasks[task_begin[b] .. task_begin[b + 1]) in order
    const int* task_begin;   // gridDim.x + 1 entries
    unsigned* abort;         // nonzero once any CTA gave up (zeroed before the launch)
    long long spin_limit;
};

// Tile forms of the batch kernel: the (n, even/odd, two-level) instantiations that
// contour_alt_kernel_for selects, in this order.
enum TeamForm {
    kTeam64EO2 = 0,
    kTeam16EO, kTeam32EO, kTeam48EO, kTeam64EO,
    kTeam8, kTeam16, kTeam24, kTeam32, kTeam40, kTeam48, kTeam56,
    kTeamForms
};

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The tensor maps of a TeamChain live in global memory (written by the host before the
// launch); order their generic-proxy contents before the bulk-copy engine reads them.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* m) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(m) : "memory");
}

// Run one task: this CTA's units of chain ch, as rank `rank` of a team of T CTAs.
// Returns false after an error (the CTA then stops taking tasks).
template <int N, bool EO, bool EO2>
__device__ bool team_chain(const BatchContourArgs& a, const TeamChain* ch, int rank, int T, double* smem,
                           unsigned long long* bar, unsigned& wpar, int* s_fail) {
    using S = AltShape<N, EO, EO2>;
    constexpr int LF = S::LF;
    constexpr int OFFY = S::AX;
    constexpr int OFFZ = 2 * S::AX;
    constexpr unsigned TILE_BYTES = N * N * sizeof(double);
    constexpr long long M = (long long)N * N * N;
    constexpr long long PLANE = (long long)N * N;
    double* sops = smem;
    double* T0 = smem + S::OPS_PAD;
    double* T1 = T0 + S::TILE;
    double* W0 = T1 + S::TILE;
    double* W1 = W0 + S::WT;
    double* QS = W1 + S::WT;
    const int warp = threadIdx.x >> 5;
    const int P = N / T;  // units of this CTA per phase (the host guarantees T | N)

    unsigned* err = ch->error;
    {
        const void* tiles[3] = {W0, W1, QS};
        const int e = tma_alignment_error(tiles, 3, ch->tm_q, 2) | tma_alignment_error(tiles, 0, &ch->tm_w[0][0], 4);
        if (e) {
            if (threadIdx.x == 0) {
                atomicOr(err, (unsigned)e);
                atomicOr(a.abort, 1u);
            }
            return false;  // the kernel lets the earlier tasks' q stores finish before it leaves
        }
    }
    if (threadIdx.x == 0) {
        tensormap_acquire(&ch->tm_q[0]);
        tensormap_acquire(&ch->tm_q[1]);
        for (int b = 0; b < 2; ++b)
            for (int v = 0; v < 2; ++v) tensormap_acquire(&ch->tm_w[b][v]);
    }
    __syncthreads();  // every thread is done with the previous task's operators
    op_copy_async(sops, ch->ops, S::OPS);
    cp_async_wait_all();
    __syncthreads();

    const int U = ch->U;
    const int dir = ch->dir;
    const long long slot0 = ch->slot0;
    const long long NsA = ch->NsA;
    double* q = ch->q;
    double* XP = ch->xbuf;  // written by plane phases
    double* XS = XP + M;    // written by slab phases
    // flags[layout][consumer CTA][producer CTA] (T x T each): phase + 1 once the producer's
    // units of that phase are in the exchange buffer
    unsigned* fl_plane = ch->flags;       // written after plane phases
    unsigned* fl_slab = fl_plane + T * T; // written after slab phases

    auto blk_of = [&](int s) -> int {
        const long long in_slot = slot0 + (long long)dir * s;
        const long long seg = dir > 0 ? in_slot : in_slot - 1;
        return seg < NsA ? 0 : 1;
    };
    // warp 0: bulk-load the Boltzmann tiles of unit p in phase k
    auto issue_w = [&](int k, int p) {
        const bool plane = (k & 1) == 0;
        const unsigned bytes = ((k >= 1) + (k < U)) * TILE_BYTES;
        if ((threadIdx.x & 31) == 0) mbar_expect_tx(bar, bytes);
        __syncwarp();
        if ((threadIdx.x & 31) == 0) {
            if (k >= 1) tma_load_4d(W0, &ch->tm_w[blk_of(k - 1)][plane ? 0 : 1], 0, 0, 0, p, bar);
            if (k < U) tma_load_4d(W1, &ch->tm_w[blk_of(k)][plane ? 0 : 1], 0, 0, 0, p, bar);
        }
    };
    auto fail_exit = [&](unsigned bits, bool w_pending) {
        if (threadIdx.x == 0) {
            atomicOr(err, bits);
            atomicOr(a.abort, 1u);
        }
        if (w_pending) mbar_wait(bar, wpar, kDrainSpins);
        if (warp == 0) bulk_wait_all();
        return false;
    };
    auto row_z = [&](const double* F, double* G) {
        if constexpr (EO2) row_op_eo2<N, N, LF>(F, G, sops + OFFZ);
        else row_op_ct<N, N, LF, EO>(F, G, sops + OFFZ);
    };
    auto col_global = [&](const double* F, const ColOut& o, int off) {
        if constexpr (EO2) col_op_eo2<N, N, LF, kToGlobal>(F, o, sops + off);
        else col_op_ct<N, N, LF, EO, kToGlobal>(F, o, sops + off);
    };

    // unit j's tile of phase k into its work tile (T0 for even j, T1 for odd j: a unit's
    // second work tile is free once its finishing operation has run, and takes the next
    // unit's tile): the contour store's input slice in phase 0, else the rows the other
    // layout wrote to its exchange buffer in phase k-1
    auto fetch = [&](int k, int j) {
        const bool plane = (k & 1) == 0;
        const int p = rank + j * T;
        const long long off = plane ? (long long)p * PLANE : (long long)p * N;
        const long long gs = plane ? N : PLANE;
        tile_fetch<N, LF>((j & 1) ? T1 : T0, (k == 0 ? q + slot0 * M : (plane ? XS : XP)) + off, gs);
        cp_async_commit();
    };

    if (warp == 0) issue_w(0, rank);
    for (int k = 0; k <= U; ++k) {
        const bool plane = (k & 1) == 0;
        if (k >= 1) {
            // every CTA of the team has finished phase k-1 (all its units written to the
            // exchange buffer): one flag per producer CTA, polled by thread t
            if (threadIdx.x < T) {
                const unsigned* f = (plane ? fl_slab : fl_plane) + (size_t)rank * T + threadIdx.x;
                long long spins = 0;
                while (ld_acquire_u32(f) < (unsigned)k) {
                    if (++spins > a.spin_limit) {
                        *s_fail = 1;
                        break;
                    }
                    if (spins > 64) {
                        if ((spins & 255) == 0 && ld_relaxed_u32(a.abort)) {
                            *s_fail = 1;
                            break;
                        }
                        __nanosleep(20);
                    }
                }
            }
            __syncthreads();
            if (*s_fail) return fail_exit(1u, true);
        }
        fetch(k, 0);
        for (int j = 0; j < P; ++j) {
            const int p = rank + j * T;
            const long long off = plane ? (long long)p * PLANE : (long long)p * N;
            const long long gs = plane ? N : PLANE;
            const bool more = j + 1 < P;  // prefetch unit j+1 into `oth` once it is free
            cp_async_wait_all();
            __syncthreads();
            double* cur = (j & 1) ? T1 : T0;
            double* oth = (j & 1) ? T0 : T1;
            if (k >= 1) {
                // finish step k-1 on this unit (A_z, then the layout's column axis, whose
                // epilogue applies D, writes q(s+1) to the staging tile and D q(s+1) to cur),
                // as contour_alt_kernel
                row_z(cur, oth);
                if (warp == 0) bulk_wait_read();  // the previous q store has left QS
                if (!mbar_wait(bar, wpar, a.spin_limit)) *s_fail = 1;
                __syncthreads();
                if (*s_fail) return fail_exit(2u, true);
                wpar ^= 1u;
                ColOut fo{cur, 0};
                fo.w0 = W0;
                fo.w1 = W1;
                fo.qs = QS;
                fo.start = k < U;
                if constexpr (EO2) col_op_eo2<N, N, LF, kFinish>(oth, fo, sops + (plane ? OFFY : 0));
                else col_op_ct<N, N, LF, EO, kFinish>(oth, fo, sops + (plane ? OFFY : 0));
                fence_async_smem();
                __syncthreads();
                if (threadIdx.x == 0) {
                    tma_store_5d(&ch->tm_q[plane ? 0 : 1], QS, 0, 0, 0, p, (int)(slot0 + (long long)dir * k));
                    bulk_commit();
                }
            } else {
                if (!mbar_wait(bar, wpar, a.spin_limit)) *s_fail = 1;
                __syncthreads();
                if (*s_fail) return fail_exit(2u, true);
                wpar ^= 1u;
                tile_scale_panel<N, LF>(cur, W1);
                __syncthreads();
            }
            if (more) fetch(k, j + 1);  // into oth, which nothing reads any more this unit
            // W0/W1 are free: prefetch the factors of the next (phase, unit)
            if (warp == 0) {
                if (more) issue_w(k, p + T);
                else if (k < U) issue_w(k + 1, rank);
            }
            if (k < U) {
                // start step k on this unit with the layout's column axis; the epilogue
                // writes the exchange buffer
                const ColOut xo{(plane ? XP : XS) + off, gs};
                col_global(cur, xo, plane ? OFFY : 0);
            }
        }
        __syncthreads();
        if (k < U && threadIdx.x < T) {  // tell CTA threadIdx.x that this CTA's units of phase k are out
            __threadfence();
            st_release_u32((plane ? fl_plane : fl_slab) + (size_t)threadIdx.x * T + rank, (unsigned)(k + 1));
        }
    }
    return true;
}

__global__ void __launch_bounds__(kContourThreads, 1) batch_contour_kernel(const __grid_constant__ BatchContourArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double* smem = reinterpret_cast<double*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
    __shared__ __align__(8) unsigned long long s_bar;  // completion of the Boltzmann tile loads
    __shared__ int s_fail;
    if (threadIdx.x == 0) {
        s_fail = 0;
        mbar_init(&s_bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned wpar = 0;
    const int t0 = a.task_begin[blockIdx.x], t1 = a.task_begin[blockIdx.x + 1];
    for (int t = t0; t < t1; ++t) {
        const TeamTask task = a.tasks[t];
        const TeamChain* ch = a.chains + task.chain;
        bool ok = false;
        switch (ch->form) {
            case kTeam64EO2: ok = team_chain<64, true, true>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam16EO: ok = team_chain<16, true, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam32EO: ok = team_chain<32, true, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam48EO: ok = team_chain<48, true, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam64EO: ok = team_chain<64, true, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam8: ok = team_chain<8, false, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam16: ok = team_chain<16, false, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam24: ok = team_chain<24, false, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam32: ok = team_chain<32, false, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam40: ok = team_chain<40, false, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam48: ok = team_chain<48, false, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            case kTeam56: ok = team_chain<56, false, false>(a, ch, task.rank, task.size, smem, &s_bar, wpar, &s_fail); break;
            default:
                if (threadIdx.x == 0) {
                    atomicOr(ch->error, 4u);
                    atomicOr(a.abort, 1u);
                }
                break;
        }
        if (!ok) break;
    }
    // the q stores of the last tasks (or of the tasks before a failure) read shared memory
    // until they complete: wait for them before the block leaves
    if ((threadIdx.x >> 5) == 0) bulk_wait_all();
}

// Dynamic shared memory the batch kernel needs for tile form f.
inline size_t team_form_smem(int f) {
    switch (f) {
        case kTeam64EO2: return AltShape<64, true, true>::SMEM;
        case kTeam16EO: return AltShape<16, true>::SMEM;
        case kTeam32EO: return AltShape<32, true>::SMEM;
        case kTeam48EO: return AltShape<48, true>::SMEM;
        case kTeam64EO: return AltShape<64, true>::SMEM;
        case kTeam8: return AltShape<8, false>::SMEM;
        case kTeam16: return AltShape<16, false>::SMEM;
        case kTeam24: return AltShape<24, false>::SMEM;
        case kTeam32: return AltShape<32, false>::SMEM;
        case kTeam40: return AltShape<40, false>::SMEM;
        case kTeam48: return AltShape<48, false>::SMEM;
        case kTeam56: return AltShape<56, false>::SMEM;
        default: return 0;
    }
}

// Tile form of a cubic grid of side n with the even/odd choice of the per-instance
// alternating kernel (contour_alt_kernel_for); -1 if the batch kernel has none.
inline int team_form_for(int n, bool eo, bool eo2) {
    if (eo2) return (eo && n == 64) ? kTeam64EO2 : -1;
    if (eo) {
        switch (n) {
            case 16: return kTeam16EO;
            case 32: return kTeam32EO;
            case 48: return kTeam48EO;
            case 64: return kTeam64EO;
            default: return -1;
        }
    }
    switch (n) {
        case 8: return kTeam8;
        case 16: return kTeam16;
        case 24: return kTeam24;
        case 32: return kTeam32;
        case 40: return kTeam40;
        case 48: return kTeam48;
        case 56: return kTeam56;
        default: return -1;
    }
}

}  // namespace crysscft
