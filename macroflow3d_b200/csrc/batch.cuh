// batch.cuh -- batched ensemble solves: many independent realisations, each on its own grid,
// solved together (included at the end of solver.cu).
//
// The reference solves an ensemble one realisation at a time: run_ensemble calls solve_head
// in its realisation loop (src/runtime/ensemble/EnsembleRunner.cu:259-317), and every solve
// is its own chain of small launches with blocking reductions.  A batch here keeps one
// HeadSolver per realisation (hierarchy, coefficients, vectors, PCG state) and replaces the
// per-realisation launch chains by batched launches over all realisations:
//   - one launch per V-cycle sweep position (level depth, pre/post, sweep index), whose
//     persistent CTAs walk the (tile, z chunk) work items of every realisation that has that
//     level; realisations whose level is not TMA-aligned (or all of them, if the tuner says
//     so) go to the L1-path sweep in a second launch;
//   - one launch for every realisation's coarse tail (one CTA each);
//   - one launch per PCG kernel;
// all of it captured once in a CUDA graph with a device `while` node.  Each realisation has
// its own stopping test; a realisation that has converged sets its stop flag and every later
// launch skips its work (the per-realisation convergence mask), and the loop ends when no
// realisation is running.  The z depth of the sweep work items (and the choice between the
// staged and the L1 sweep) is picked per sweep position by an autotuner that times the
// candidates on the batch itself.
#pragma once
#include "kernels_batch.cuh"

namespace mf3d {

// cudaOccupancy for a batched staged sweep (and its shared-memory attributes)
template <class T, class TC, int MODE> static int tma_batch_setup() {
    using C = TmaSweepCfg<T, TC, MODE>;
    MF3D_CK(cudaFuncSetAttribute(sweep_tma_kernel<T, TC, MODE, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)C::SMEM));
    MF3D_CK(cudaFuncSetAttribute(sweep_tma_kernel<T, TC, MODE, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
    int n = 0;
    MF3D_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_tma_kernel<T, TC, MODE, true>, C::NT, C::SMEM));
    if (n < 1) throw Error(MF3D_E_CUDA, "staged sweep does not fit on an SM");
    return n;
}

// dynamic shared memory and resident CTAs per SM of a batched x-pair sweep (TMA form)
template <class T, class TC, int MODE> static int pair_batch_setup() {
    const size_t smem = sp_smem_bytes<T, TC, true>();
    MF3D_CK(cudaFuncSetAttribute(sweep_pair_kernel<T, TC, MODE, true, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MF3D_CK(cudaFuncSetAttribute(sweep_pair_kernel<T, TC, MODE, true, true>,
                                 cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
    int n = 0;
    MF3D_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_pair_kernel<T, TC, MODE, true, true>, SP_NT, smem));
    if (n < 1) throw Error(MF3D_E_CUDA, "x-pair sweep does not fit on an SM");
    return n;
}

class BatchSolverBase {
  public:
    virtual ~BatchSolverBase() {}
    virtual void set_K(const double* const* K) = 0;
    virtual void solve(double* const* h, const double* const* x0, mf3d_solve_result* res) = 0;
    virtual std::vector<mf3d_batch_tuning> autotune(int reps) = 0;
    virtual long long device_bytes() const = 0;
    virtual int count() const = 0;
};

// host-side layout of a small device table: appends arrays at 256-byte boundaries
struct Blob {
    std::vector<unsigned char> h;
    size_t add(const void* src, size_t bytes) {
        const size_t off = (h.size() + 255) & ~(size_t)255;
        h.resize(off + bytes);
        if (src && bytes) std::memcpy(h.data() + off, src, bytes);
        return off;
    }
    std::unique_ptr<DevMem> upload() const {
        std::unique_ptr<DevMem> m(new DevMem(std::max<size_t>(h.size(), 256)));
        if (!h.empty()) MF3D_CK(cudaMemcpy(m->p, h.data(), h.size(), cudaMemcpyHostToDevice));
        return m;
    }
};

template <class T, class TC> class BatchSolverT : public BatchSolverBase {
    using VC = VCycle<T, TC>;
    using Rec = typename VC::RecSweep;
    // The batched x-pair sweep (path 2) is kept off: default bench runs that used it, with the
    // batched residual + restriction after it, stopped with an illegal address or stalled
    // TMA waits in the ensemble's autotuner, in a process that had run other solves first,
    // and the cause is not found.  Batched solves use the staged quad sweep and the L1 sweep.
    static constexpr bool kPairPath = false;

    // one batched launch of a sweep position: x-pair (TMA), staged quad (TMA) or L1 form; or
    // of a residual + restriction position
    struct Launch {
        bool rr = false;
        const RrItem<T, TC>* ritems = nullptr;
        const int* roff = nullptr;
        bool pair = false;
        SpArgs<T, TC> pa0{}; // x-pair: the launch-wide argument
        bool tma = false;
        int nseg = 0, total = 0;
        unsigned grid = 0;
        std::unique_ptr<DevMem> mem;
        TmaSweepArgs<T, TC> a0{};                   // staged: the launch-wide argument
        const SweepArgs<T, TC, T>* largs = nullptr; // L1: per-segment arguments, grids, offsets
        const int4* ldims = nullptr;
        const int* loff = nullptr;
    };
    // one sweep position of the V-cycle, over every realisation that has that level
    struct Op {
        int phase, level, sw, mode;
        std::vector<int> real; // realisation of each record
        std::vector<Rec> rec;
        // 0: staged quad where aligned, 1: L1 only, 2: x-pair where it serves (else as 0);
        // z chunks per tile
        int path = 0, chunks = 1;
        std::vector<Launch> launches;
    };

  public:
    BatchSolverT(std::vector<std::unique_ptr<HeadSolver>>&& hs, const mf3d_solver_config& cfg, cudaStream_t s,
                 cudaStream_t own)
        : hs_(std::move(hs)), cfg_(cfg), s_(s), own_stream_(own) {
        const int R = (int)hs_.size();
        occ_[0] = tma_batch_setup<T, TC, 0>();
        occ_[M_ZERO] = tma_batch_setup<T, TC, M_ZERO>();
        occ_[M_PROLONG] = tma_batch_setup<T, TC, M_PROLONG>();
        occ_[M_ZERO | M_PROLONG] = tma_batch_setup<T, TC, M_ZERO | M_PROLONG>();
        occ_[M_RESID] = tma_batch_setup<T, TC, M_RESID>();
        occ_[M_ZERO | M_RESID] = tma_batch_setup<T, TC, M_ZERO | M_RESID>();
        occ_[M_DOT] = tma_batch_setup<T, TC, M_DOT>();
        occ_[M_ZERO | M_DOT] = tma_batch_setup<T, TC, M_ZERO | M_DOT>();
        occ_[M_PROLONG | M_DOT] = tma_batch_setup<T, TC, M_PROLONG | M_DOT>();
        occ_[M_ZERO | M_PROLONG | M_DOT] = tma_batch_setup<T, TC, M_ZERO | M_PROLONG | M_DOT>();
        MF3D_CK(cudaFuncSetAttribute(resid_restrict_batch_kernel<T, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)rr_smem_bytes<T, TC>()));
        if constexpr (VC::kPair && kPairPath) {
            pocc_[0] = pair_batch_setup<T, TC, 0>();
            pocc_[M_ZERO] = pair_batch_setup<T, TC, M_ZERO>();
            pocc_[M_PROLONG] = pair_batch_setup<T, TC, M_PROLONG>();
            pocc_[M_ZERO | M_PROLONG] = pair_batch_setup<T, TC, M_ZERO | M_PROLONG>();
            pocc_[M_DOT] = pair_batch_setup<T, TC, M_DOT>();
            pocc_[M_ZERO | M_DOT] = pair_batch_setup<T, TC, M_ZERO | M_DOT>();
            pocc_[M_PROLONG | M_DOT] = pair_batch_setup<T, TC, M_PROLONG | M_DOT>();
            pocc_[M_ZERO | M_PROLONG | M_DOT] = pair_batch_setup<T, TC, M_ZERO | M_PROLONG | M_DOT>();
        }

        // ---- record every realisation's V-cycle ----
        std::vector<std::vector<Rec>> recs(R);
        std::vector<typename VC::RecTail> tails(R);
        for (int r = 0; r < R; ++r) {
            HeadSolver& H = *hs_[r];
            VC* vc = dynamic_cast<VC*>(H.vc_.get());
            if (!vc) throw Error(MF3D_E_INVALID, "batched solve: V-cycle type mismatch");
            if (vc->levels_above_tail() < 1)
                throw Error(MF3D_E_INVALID, "batched solve: every grid needs a level above the coarse tail");
            vc->rec_ = &recs[r];
            vc->rec_tail_ = &tails[r];
            try {
                vc->run(nullptr, H.z_.p, &H.state_.as<PcgState>()->rho_new);
            } catch (...) {
                vc->rec_ = nullptr;
                vc->rec_tail_ = nullptr;
                throw;
            }
            vc->rec_ = nullptr;
            vc->rec_tail_ = nullptr;
        }
        // ---- group the sweeps by position: down (level up, sweep up), then up (level down) ----
        for (int phase = 0; phase < 2; ++phase) {
            std::vector<Op> ops;
            for (int r = 0; r < R; ++r)
                for (const Rec& x : recs[r]) {
                    if (x.phase != phase) continue;
                    // one launch per position and mode: a position's last pre-sweep is the fused
                    // RESID sweep for some realisations and a sweep followed by its own residual +
                    // restriction (sw + 1) for others
                    Op* op = nullptr;
                    for (Op& o : ops)
                        if (o.level == x.level && o.sw == x.sw && o.mode == x.mode) op = &o;
                    if (!op) {
                        ops.push_back(Op{});
                        op = &ops.back();
                        op->phase = phase;
                        op->level = x.level;
                        op->sw = x.sw;
                        op->mode = x.mode;
                    }
                    if (op->mode != x.mode) throw Error(MF3D_E_INVALID, "batched solve: sweep modes differ");
                    op->real.push_back(r);
                    op->rec.push_back(x);
                }
            std::sort(ops.begin(), ops.end(), [&](const Op& a, const Op& b) {
                if (a.level != b.level) return phase == 0 ? a.level < b.level : a.level > b.level;
                return a.sw < b.sw;
            });
            for (Op& o : ops) ops_.push_back(std::move(o));
        }
        for (Op& o : ops_) {
            default_choice(o);
            o.launches = build(o, o.path, o.chunks);
        }
        // ---- coarse tails ----
        {
            std::vector<TailItem<T, T>> items(R);
            for (int r = 0; r < R; ++r) {
                items[r].a = tails[r].a;
                items[r].b_in = tails[r].b;
                items[r].x_out = tails[r].out;
                items[r].stop = &hs_[r]->state_.as<PcgState>()->stop;
                tail_smem_ = std::max(tail_smem_, tails[r].smem);
            }
            Blob b;
            b.add(items.data(), items.size() * sizeof(items[0]));
            tail_mem_ = b.upload();
            // largest tail of any batch (the attribute is the kernel's, shared by all batches)
            MF3D_CK(cudaFuncSetAttribute(tail2_batch_kernel<T, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTailSmemMax));
        }
        // ---- PCG items and the launch tables of the cell and streaming kernels ----
        {
            std::vector<PcgItem> items(R);
            std::vector<int> off3(R + 1, 0), off1(R + 1, 0);
            for (int r = 0; r < R; ++r) {
                HeadSolver& H = *hs_[r];
                PcgItem& it = items[r];
                it.L = H.op64_[0];
                it.x = H.x_.as<double>();
                it.b = H.b_.as<double>();
                it.r = H.r_.as<double>();
                it.p = H.p_.as<double>();
                it.p2 = H.p2_.as<double>();
                it.Ap = H.Ap_.as<double>();
                it.z = H.z_.p;
                it.r32 = H.r32_.as<float>();
                it.st = H.state_.as<PcgState>();
                it.partials = H.partials_.as<double>();
                it.tickets = H.tickets_.as<unsigned>();
                it.err = H.err_.as<int>();
                it.n = H.G_[0].n;
                const ColLaunch cl = col_launch(H.G_[0].nx, H.G_[0].ny, H.G_[0].nz);
                it.zchunk = cl.zchunk;
                it.cgx = (int)cl.grid.x;
                it.cgy = (int)cl.grid.y;
                it.cgz = (int)cl.grid.z;
                it.n1 = (int)grid1d(it.n, PK_NT);
                off3[r + 1] = off3[r] + (int)cl.nblocks;
                off1[r + 1] = off1[r] + it.n1;
            }
            tot3_ = off3[R];
            tot1_ = off1[R];
            Blob b;
            const size_t oi = b.add(items.data(), items.size() * sizeof(PcgItem));
            const size_t o3 = b.add(off3.data(), off3.size() * sizeof(int));
            const size_t o1 = b.add(off1.data(), off1.size() * sizeof(int));
            const size_t oc = b.add(nullptr, 2 * R * sizeof(CopyItem));
            const size_t ost = b.add(nullptr, R * (sizeof(PcgState) + sizeof(int))); // states, then error flags
            const size_t octl = b.add(nullptr, sizeof(BatchCtl) + 16);
            pcg_mem_ = b.upload();
            unsigned char* base = pcg_mem_->as<unsigned char>();
            items_d_ = reinterpret_cast<PcgItem*>(base + oi);
            off3_d_ = reinterpret_cast<int*>(base + o3);
            off1_d_ = reinterpret_cast<int*>(base + o1);
            copy_d_ = reinterpret_cast<CopyItem*>(base + oc);
            states_d_ = reinterpret_cast<PcgState*>(base + ost);
            errs_d_ = reinterpret_cast<int*>(states_d_ + R);
            ctl_d_ = reinterpret_cast<BatchCtl*>(base + octl);
            any_d_ = reinterpret_cast<int*>(base + octl + sizeof(BatchCtl));
        }
        MF3D_CK(cudaMallocHost(&copy_h_, 2 * R * sizeof(CopyItem)));
        MF3D_CK(cudaMallocHost(&states_h_, R * sizeof(PcgState) + R * sizeof(int) + 16));
        MF3D_CK(cudaEventCreate(&ev0_));
        MF3D_CK(cudaEventCreate(&ev1_));
        flexible_ = cfg.flexible < 0 ? (cfg.precision != MF3D_PREC_FP64) : (cfg.flexible != 0);
    }

    ~BatchSolverT() override {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (graph_) cudaGraphDestroy(graph_);
        if (copy_h_) cudaFreeHost(copy_h_);
        if (states_h_) cudaFreeHost(states_h_);
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        if (own_stream_) cudaStreamSynchronize(own_stream_);
        hs_.clear();
        if (own_stream_) cudaStreamDestroy(own_stream_);
    }

    int count() const override { return (int)hs_.size(); }

    long long device_bytes() const override {
        long long b = 0;
        for (const auto& h : hs_) b += h->device_bytes();
        for (const Op& o : ops_)
            for (const Launch& l : o.launches) b += (long long)l.mem->bytes;
        for (const auto& m : retired_) b += (long long)m->bytes;
        return b + (long long)tail_mem_->bytes + (long long)pcg_mem_->bytes;
    }

    void set_K(const double* const* K) override {
        for (size_t r = 0; r < hs_.size(); ++r) hs_[r]->set_K(K[r]);
    }

    void solve(double* const* h, const double* const* x0, mf3d_solve_result* res) override {
        const int R = (int)hs_.size();
        for (int r = 0; r < R; ++r) {
            if (!hs_[r]->have_K_) throw Error(MF3D_E_STATE, "set_K must be called before solve");
            if (!h[r]) throw Error(MF3D_E_INVALID, "h is null");
        }
        const long long l0 = g_launches;
        for (int r = 0; r < R; ++r) {
            HeadSolver& H = *hs_[r];
            copy_h_[r] = CopyItem{(x0 && x0[r]) ? x0[r] : H.x0_.as<double>(), H.x_.as<double>(), H.G_[0].n};
            copy_h_[R + r] = CopyItem{H.x_.as<double>(), h[r], H.G_[0].n};
        }
        MF3D_CK(cudaEventRecord(ev0_, s_));
        MF3D_CK(cudaMemcpyAsync(copy_d_, copy_h_, 2 * R * sizeof(CopyItem), cudaMemcpyHostToDevice, s_));
        long long bodies = 0;
        (void)bodies;
        if (cfg_.use_graph) {
            if (!exec_) build_graph();
            MF3D_CK(cudaGraphLaunch(exec_, s_));
        } else {
            // host-driven loop (profilers): the same launches, the gate's flag polled each time
            int* any_h = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(states_h_) + R * sizeof(PcgState) +
                                                R * sizeof(int));
            record_pre(s_, false);
            for (int it = 0; it <= cfg_.cg_max_iter + 1; ++it) {
                MF3D_CK(cudaMemcpyAsync(any_h, any_d_, sizeof(int), cudaMemcpyDeviceToHost, s_));
                MF3D_CK(cudaStreamSynchronize(s_));
                if (!*any_h) break;
                record_body(s_, false);
                ++bodies;
            }
            record_post(s_);
        }
        MF3D_CK(cudaEventRecord(ev1_, s_));
        MF3D_CK(cudaMemcpyAsync(states_h_, states_d_, R * (sizeof(PcgState) + sizeof(int)), cudaMemcpyDeviceToHost,
                                s_));
        MF3D_CK(cudaStreamSynchronize(s_));
        const PcgState* st = states_h_;
        const int* errs = reinterpret_cast<const int*>(states_h_ + R);
        for (int r = 0; r < R; ++r)
            if (errs[r]) throw Error(MF3D_E_CUDA, "a TMA pipeline wait timed out in the smoother");
        long long launches = g_launches - l0;
        if (cfg_.use_graph) {
            int maxit = 0;
            for (int r = 0; r < R; ++r) maxit = std::max(maxit, st[r].iter);
            launches += pre_launches_ + post_launches_ + (long long)maxit * body_launches_;
        }
        float ms = 0.f;
        MF3D_CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
        if (res)
            for (int r = 0; r < R; ++r) {
                mf3d_solve_result& o = res[r];
                std::memset(&o, 0, sizeof(o));
                o.num_iterations = st[r].iter;
                o.converged = st[r].converged;
                o.status = st[r].status;
                o.num_levels = hs_[r]->num_levels();
                o.initial_residual = std::sqrt(st[r].r0sq);
                o.final_residual = st[r].final_res;
                o.b_norm = std::sqrt(st[r].bb);
                o.true_rel_residual = st[r].bb > 0 ? std::sqrt(st[r].rr_true / st[r].bb) : std::sqrt(st[r].rr_true);
                o.device_ms = ms;
                o.kernel_launches = (int)launches;
            }
    }

    // Times every candidate of every sweep position (reps launches each, after one warm-up)
    // and keeps the fastest; the solver's state is scratch afterwards.
    std::vector<mf3d_batch_tuning> autotune(int reps) override {
        reps = std::max(1, reps);
        const int R = (int)hs_.size();
        batch_init_kernel<<<1, 256, 0, s_>>>(items_d_, R, ctl_d_, 1, 1, 0, 0.0, kSolveBudgetNs, SOLVE_PCG_MG, 1);
        MF3D_LAUNCH_CK();
        std::vector<mf3d_batch_tuning> out;
        for (Op& o : ops_) {
            mf3d_batch_tuning t{};
            t.phase = o.phase;
            t.level = o.level;
            t.sweep = o.sw;
            t.mode = o.mode;
            t.ms_default = time_launches(o.mode, o.launches, reps);
            if (o.rec[0].kind == 1) { // residual + restriction: one shape
                t.path = o.path;
                t.chunks = o.chunks;
                t.ms_best = t.ms_default;
                out.push_back(t);
                continue;
            }
            int best_path = o.path, best_chunks = o.chunks;
            double best = t.ms_default;
            bool any_tma = false, any_pair = false;
            int nzmin = 1 << 30;
            for (const Rec& x : o.rec) {
                any_tma |= x.tma;
                any_pair |= x.pair;
                nzmin = std::min(nzmin, x.g.nz);
            }
            for (int path = any_tma ? 0 : 1; path < (kPairPath && any_pair ? 3 : 2); ++path)
                for (int chunks = 1; chunks <= 8 && (chunks == 1 || 2 * chunks <= nzmin); chunks *= 2) {
                    if (path == o.path && chunks == o.chunks) continue;
                    std::vector<Launch> cand = build(o, path, chunks);
                    const double ms = time_launches(o.mode, cand, reps);
                    retire(cand);
                    if (ms < best) {
                        best = ms;
                        best_path = path;
                        best_chunks = chunks;
                    }
                }
            if (best_path != o.path || best_chunks != o.chunks) {
                o.path = best_path;
                o.chunks = best_chunks;
                retire(o.launches);
                o.launches = build(o, o.path, o.chunks);
            }
            t.path = o.path;
            t.chunks = o.chunks;
            t.ms_best = best;
            out.push_back(t);
        }
        MF3D_CK(cudaStreamSynchronize(s_));
        // the graph holds the launches of the previous choice
        if (exec_) cudaGraphExecDestroy(exec_);
        if (graph_) cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
        return out;
    }

  private:
    void default_choice(Op& o) {
        bool any_tma = false, any_pair = false;
        long long tiles = 0, cols = 0, ptiles = 0;
        for (const Rec& x : o.rec) {
            any_tma |= x.tma;
            any_pair |= x.pair;
            const int TX = TmaSweepCfg<T, TC, 0>::TX, TY = TmaSweepCfg<T, TC, 0>::TY;
            if (x.tma) tiles += (long long)((x.g.nx + TX - 1) / TX) * ((x.g.ny + TY - 1) / TY);
            if (x.pair) ptiles += (long long)((x.g.nx + pair_tx() - 1) / pair_tx()) * ((x.g.ny + SP_TY - 1) / SP_TY);
            cols += (long long)((x.g.nx + SW_TX - 1) / SW_TX) * ((x.g.ny + SW_TY - 1) / SW_TY);
        }
        o.path = kPairPath && any_pair ? 2 : (any_tma ? 0 : 1);
        if (o.path == 2) {
            const long long resident = (long long)std::max(1, pocc_[o.mode & 15]) * num_sms();
            o.chunks = (int)std::max<long long>(1, std::min<long long>(8, resident / std::max(1LL, ptiles)));
        } else if (o.path == 0) {
            const long long resident = (long long)std::max(1, occ_[o.mode & 15]) * num_sms();
            o.chunks = (int)std::max<long long>(1, std::min<long long>(8, resident / std::max(1LL, tiles)));
        } else {
            o.chunks = (int)std::max<long long>(1, std::min<long long>(16, (long long)num_sms() * 6 / std::max(1LL, cols)));
        }
    }

    static int chunk_planes(int nz, int chunks) {
        const int nc = std::max(1, std::min(chunks, std::max(1, nz / 2)));
        return 2 * (((nz + 1) / 2 + nc - 1) / nc);
    }

    // the launches of sweep position o for a choice: the staged sweep for the realisations
    // whose level has a staged form (path 0), the L1 sweep for the others
    static constexpr int pair_tx() { return sp_tx<T, TC, true>(); }

    std::vector<Launch> build(const Op& o, int path, int chunks) const {
        if (o.rec[0].kind == 1) { // residual + restriction of every realisation at this position
            std::vector<int> off(1, 0);
            std::vector<RrItem<T, TC>> items;
            for (int i = 0; i < (int)o.rec.size(); ++i) {
                RrItem<T, TC> it = o.rec[i].rr;
                HeadSolver& H = *hs_[o.real[i]];
                it.stop = &H.state_.as<PcgState>()->stop;
                off.push_back(off.back() + it.gx * it.gy * it.gz);
                items.push_back(it);
            }
            Blob b;
            const size_t oo = b.add(off.data(), off.size() * sizeof(int));
            const size_t oi = b.add(items.data(), items.size() * sizeof(items[0]));
            Launch L;
            L.rr = true;
            L.nseg = (int)items.size();
            L.total = off.back();
            L.grid = (unsigned)L.total;
            L.mem = b.upload();
            unsigned char* base = L.mem->template as<unsigned char>();
            L.roff = reinterpret_cast<const int*>(base + oo);
            L.ritems = reinterpret_cast<const RrItem<T, TC>*>(base + oi);
            std::vector<Launch> out;
            out.push_back(std::move(L));
            return out;
        }
        std::vector<int> ps, ts, ls;
        for (int i = 0; i < (int)o.rec.size(); ++i) {
            const Rec& x = o.rec[i];
            if (path == 2 && x.pair) ps.push_back(i);
            else if (path != 1 && x.tma) ts.push_back(i);
            else ls.push_back(i);
        }
        std::vector<Launch> out;
        if (!ps.empty()) {
            std::vector<int> off(1, 0);
            std::vector<SpArgs<T, TC>> args;
            std::vector<SpMaps> maps;
            for (int i : ps) {
                const Rec& x = o.rec[i];
                HeadSolver& H = *hs_[o.real[i]];
                SpArgs<T, TC> a = x.pa;
                a.zchunk = chunk_planes(x.g.nz, chunks);
                a.stop = &H.state_.as<PcgState>()->stop;
                const int ntiles = ((x.g.nx + pair_tx() - 1) / pair_tx()) * ((x.g.ny + SP_TY - 1) / SP_TY);
                const int items = ntiles * ((x.g.nz + a.zchunk - 1) / a.zchunk);
                if ((o.mode & M_DOT) && (size_t)items > vc_of(o.real[i])->scratch().partial_cap)
                    throw Error(MF3D_E_INVALID, "reduction scratch too small");
                off.push_back(off.back() + items);
                args.push_back(a);
                maps.push_back(*x.pmaps);
            }
            Blob b;
            const size_t oo = b.add(off.data(), off.size() * sizeof(int));
            const size_t oa = b.add(args.data(), args.size() * sizeof(args[0]));
            const size_t om = b.add(maps.data(), maps.size() * sizeof(SpMaps));
            Launch L;
            L.pair = true;
            L.nseg = (int)ps.size();
            L.total = off.back();
            L.mem = b.upload();
            unsigned char* base = L.mem->template as<unsigned char>();
            L.pa0.seg_off = reinterpret_cast<const int*>(base + oo);
            L.pa0.seg_args = reinterpret_cast<const SpArgs<T, TC>*>(base + oa);
            L.pa0.seg_maps = reinterpret_cast<const SpMaps*>(base + om);
            L.pa0.nseg = L.nseg;
            L.pa0.total = L.total;
            const long long resident = (long long)std::max(1, pocc_[o.mode & 15]) * num_sms();
            L.grid = (unsigned)std::max<long long>(1, std::min<long long>(L.total, resident));
            out.push_back(std::move(L));
        }
        if (!ts.empty()) {
            const int TX = TmaSweepCfg<T, TC, 0>::TX, TY = TmaSweepCfg<T, TC, 0>::TY;
            std::vector<int> off(1, 0);
            std::vector<TmaSweepArgs<T, TC>> args;
            std::vector<TmaMaps> maps;
            for (int i : ts) {
                const Rec& x = o.rec[i];
                HeadSolver& H = *hs_[o.real[i]];
                TmaSweepArgs<T, TC> a = x.ta;
                a.zchunk = chunk_planes(x.g.nz, chunks);
                a.stop = &H.state_.as<PcgState>()->stop;
                const int ntiles = ((x.g.nx + TX - 1) / TX) * ((x.g.ny + TY - 1) / TY);
                const int items = ntiles * ((x.g.nz + a.zchunk - 1) / a.zchunk);
                if ((o.mode & M_DOT) && (size_t)items > vc_of(o.real[i])->scratch().partial_cap)
                    throw Error(MF3D_E_INVALID, "reduction scratch too small");
                off.push_back(off.back() + items);
                args.push_back(a);
                maps.push_back(*x.maps);
            }
            Blob b;
            const size_t oo = b.add(off.data(), off.size() * sizeof(int));
            const size_t oa = b.add(args.data(), args.size() * sizeof(args[0]));
            const size_t om = b.add(maps.data(), maps.size() * sizeof(TmaMaps));
            Launch L;
            L.tma = true;
            L.nseg = (int)ts.size();
            L.total = off.back();
            L.mem = b.upload();
            unsigned char* base = L.mem->template as<unsigned char>();
            L.a0.seg_off = reinterpret_cast<const int*>(base + oo);
            L.a0.seg_args = reinterpret_cast<const TmaSweepArgs<T, TC>*>(base + oa);
            L.a0.seg_maps = reinterpret_cast<const TmaMaps*>(base + om);
            L.a0.nseg = L.nseg;
            L.a0.total = L.total;
            const long long resident = (long long)std::max(1, occ_[o.mode & 15]) * num_sms();
            L.grid = (unsigned)std::max<long long>(1, std::min<long long>(L.total, resident));
            out.push_back(std::move(L));
        }
        if (!ls.empty()) {
            std::vector<int> off(1, 0);
            std::vector<SweepArgs<T, TC, T>> args;
            std::vector<int4> dims;
            for (int i : ls) {
                const Rec& x = o.rec[i];
                HeadSolver& H = *hs_[o.real[i]];
                SweepArgs<T, TC, T> a = x.la;
                a.zchunk = chunk_planes(x.g.nz, chunks);
                a.stop = &H.state_.as<PcgState>()->stop;
                const int gx = (x.g.nx + SW_TX - 1) / SW_TX, gy = (x.g.ny + SW_TY - 1) / SW_TY;
                const int gz = (x.g.nz + a.zchunk - 1) / a.zchunk;
                if ((o.mode & M_DOT) && (size_t)gx * gy * gz > vc_of(o.real[i])->scratch().partial_cap)
                    throw Error(MF3D_E_INVALID, "reduction scratch too small");
                off.push_back(off.back() + gx * gy * gz);
                args.push_back(a);
                dims.push_back(make_int4(gx, gy, gz, 0));
            }
            Blob b;
            const size_t oo = b.add(off.data(), off.size() * sizeof(int));
            const size_t oa = b.add(args.data(), args.size() * sizeof(args[0]));
            const size_t od = b.add(dims.data(), dims.size() * sizeof(int4));
            Launch L;
            L.tma = false;
            L.nseg = (int)ls.size();
            L.total = off.back();
            L.grid = (unsigned)L.total;
            L.mem = b.upload();
            unsigned char* base = L.mem->template as<unsigned char>();
            L.loff = reinterpret_cast<const int*>(base + oo);
            L.largs = reinterpret_cast<const SweepArgs<T, TC, T>*>(base + oa);
            L.ldims = reinterpret_cast<const int4*>(base + od);
            out.push_back(std::move(L));
        }
        return out;
    }

    VC* vc_of(int r) const { return static_cast<VC*>(hs_[r]->vc_.get()); }

    // Launch tables hold tensor maps that kernels read from device memory.  A table is never
    // freed while the solver lives, so no later table (another candidate's maps) is written
    // at an address whose descriptor the TMA unit may still cache.
    void retire(std::vector<Launch>& ls) {
        for (Launch& L : ls)
            if (L.mem) retired_.push_back(std::move(L.mem));
        ls.clear();
    }

    template <int MODE> void launch_one(cudaStream_t s, const Launch& L) const {
        if (L.pair) {
            if constexpr (VC::kPair && (MODE & M_RESID) == 0) {
                sweep_pair_kernel<T, TC, MODE, true, true>
                    <<<L.grid, SP_NT, sp_smem_bytes<T, TC, true>(), s>>>(SpMaps{}, L.pa0);
            } else {
                throw Error(MF3D_E_INVALID, "x-pair sweep: unsupported batched mode");
            }
        } else if (L.tma) {
            using C = TmaSweepCfg<T, TC, MODE>;
            sweep_tma_kernel<T, TC, MODE, true><<<L.grid, C::NT, C::SMEM, s>>>(TmaMaps{}, L.a0);
        } else {
            sweep_batch_kernel<T, TC, T, MODE><<<L.grid, SW_NT, 0, s>>>(L.largs, L.ldims, L.loff, L.nseg);
        }
        MF3D_LAUNCH_CK();
    }

    void launch(cudaStream_t s, int mode, const Launch& L) const {
        if (L.rr) {
            resid_restrict_batch_kernel<T, TC><<<L.grid, 256, rr_smem_bytes<T, TC>(), s>>>(L.ritems, L.roff, L.nseg);
            MF3D_LAUNCH_CK();
            return;
        }
        switch (mode) {
        case 0: launch_one<0>(s, L); break;
        case M_ZERO: launch_one<M_ZERO>(s, L); break;
        case M_PROLONG: launch_one<M_PROLONG>(s, L); break;
        case M_ZERO | M_PROLONG: launch_one<M_ZERO | M_PROLONG>(s, L); break;
        case M_RESID: launch_one<M_RESID>(s, L); break;
        case M_ZERO | M_RESID: launch_one<M_ZERO | M_RESID>(s, L); break;
        case M_DOT: launch_one<M_DOT>(s, L); break;
        case M_ZERO | M_DOT: launch_one<M_ZERO | M_DOT>(s, L); break;
        case M_PROLONG | M_DOT: launch_one<M_PROLONG | M_DOT>(s, L); break;
        case M_ZERO | M_PROLONG | M_DOT: launch_one<M_ZERO | M_PROLONG | M_DOT>(s, L); break;
        default: throw Error(MF3D_E_INVALID, "unsupported sweep mode");
        }
    }

    // mean device time of one pass over the launches (one warm-up pass first)
    double time_launches(int mode, const std::vector<Launch>& ls, int reps) {
        for (const Launch& L : ls) launch(s_, mode, L);
        MF3D_CK(cudaEventRecord(ev0_, s_));
        for (int i = 0; i < reps; ++i)
            for (const Launch& L : ls) launch(s_, mode, L);
        MF3D_CK(cudaEventRecord(ev1_, s_));
        MF3D_CK(cudaEventSynchronize(ev1_));
        float ms = 0.f;
        MF3D_CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
        return ms / reps;
    }

    void record_vcycle(cudaStream_t s) const {
        const int R = (int)hs_.size();
        size_t i = 0;
        for (; i < ops_.size() && ops_[i].phase == 0; ++i)
            for (const Launch& L : ops_[i].launches) launch(s, ops_[i].mode, L);
        tail2_batch_kernel<T, T><<<R, TAIL2_NT, tail_smem_, s>>>(tail_mem_->as<TailItem<T, T>>());
        MF3D_LAUNCH_CK();
        for (; i < ops_.size(); ++i)
            for (const Launch& L : ops_[i].launches) launch(s, ops_[i].mode, L);
    }

    unsigned pgrid(int total) const {
        return (unsigned)std::max(1, std::min(total, num_sms() * 8));
    }

    void record_pre(cudaStream_t s, bool with_cond) {
        const int R = (int)hs_.size();
        batch_copy_kernel<<<pgrid(tot1_), PK_NT, 0, s>>>(copy_d_, off1_d_, R, tot1_);
        MF3D_LAUNCH_CK();
        batch_init_kernel<<<1, 256, 0, s>>>(items_d_, R, ctl_d_, cfg_.cg_max_iter, cfg_.cg_check_every,
                                            flexible_ ? 1 : 0, cfg_.cg_rtol, kSolveBudgetNs, SOLVE_PCG_MG,
                                            cfg_.cg_max_iter + 1);
        MF3D_LAUNCH_CK();
        batch_residual_kernel<<<pgrid(tot3_), dim3(32, 8), 0, s>>>(items_d_, off3_d_, R, tot3_, 0,
                                                                   cfg_.conv_norm == MF3D_CONV_B ? 1 : 0);
        MF3D_LAUNCH_CK();
        batch_gate_kernel<<<1, 256, 0, s>>>(items_d_, R, ctl_d_, cond_, with_cond ? 1 : 0, 0, any_d_);
        MF3D_LAUNCH_CK();
    }

    void record_body(cudaStream_t s, bool with_cond) {
        const int R = (int)hs_.size();
        record_vcycle(s);
        MF3D_CK(cudaFuncSetAttribute(batch_pmatvec_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)pmv_smem_bytes<T>()));
        batch_pmatvec_kernel<T><<<pgrid(tot3_), dim3(PMV_TX, PMV_TY), pmv_smem_bytes<T>(), s>>>(items_d_, off3_d_, R,
                                                                                             tot3_);
        MF3D_LAUNCH_CK();
        batch_xr_update_kernel<T><<<pgrid(tot1_), PK_NT, 0, s>>>(items_d_, off1_d_, R, tot1_);
        MF3D_LAUNCH_CK();
        batch_gate_kernel<<<1, 256, 0, s>>>(items_d_, R, ctl_d_, cond_, with_cond ? 1 : 0, 1, any_d_);
        MF3D_LAUNCH_CK();
    }

    void record_post(cudaStream_t s) {
        const int R = (int)hs_.size();
        batch_residual_kernel<<<pgrid(tot3_), dim3(32, 8), 0, s>>>(items_d_, off3_d_, R, tot3_, 1,
                                                                   cfg_.conv_norm == MF3D_CONV_B ? 1 : 0);
        MF3D_LAUNCH_CK();
        batch_copy_kernel<<<pgrid(tot1_), PK_NT, 0, s>>>(copy_d_ + R, off1_d_, R, tot1_);
        MF3D_LAUNCH_CK();
        batch_states_kernel<<<1, 256, 0, s>>>(items_d_, R, states_d_, errs_d_);
        MF3D_LAUNCH_CK();
    }

    // [copy in, init, residual, gate] while (any running) { V-cycle, p, Ap, x/r, gate }
    // [true residual, copy out, states], one graph
    void build_graph() {
        cudaStream_t cs = nullptr, bs = nullptr;
        MF3D_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        MF3D_CK(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
        const long long l0 = g_launches;
        bool capturing = false, capturing_body = false;
        try {
            MF3D_CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            capturing = true;
            cudaStreamCaptureStatus status;
            cudaGraph_t g = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            MF3D_CK(cudaStreamGetCaptureInfo(cs, &status, nullptr, &g, &deps, &nd));
            MF3D_CK(cudaGraphConditionalHandleCreate(&cond_, g, 0u, cudaGraphCondAssignDefault));
            record_pre(cs, true);
            pre_launches_ = (int)(g_launches - l0);
            MF3D_CK(cudaStreamGetCaptureInfo(cs, &status, nullptr, &g, &deps, &nd));
            cudaGraphNodeParams cp{};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond_;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            MF3D_CK(cudaGraphAddNode(&node, g, deps, nd, &cp));
            MF3D_CK(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
            const long long l1 = g_launches;
            MF3D_CK(cudaStreamBeginCaptureToGraph(bs, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal));
            capturing_body = true;
            record_body(bs, true);
            cudaGraph_t tmp;
            capturing_body = false;
            MF3D_CK(cudaStreamEndCapture(bs, &tmp));
            body_launches_ = (int)(g_launches - l1);
            const long long l2 = g_launches;
            record_post(cs);
            post_launches_ = (int)(g_launches - l2);
            capturing = false;
            MF3D_CK(cudaStreamEndCapture(cs, &graph_));
        } catch (...) {
            cudaGraph_t tmp;
            if (capturing_body) cudaStreamEndCapture(bs, &tmp);
            if (capturing) cudaStreamEndCapture(cs, &tmp);
            cudaStreamDestroy(cs);
            cudaStreamDestroy(bs);
            g_launches = l0;
            throw;
        }
        g_launches = l0; // captured, not launched
        MF3D_CK(cudaStreamDestroy(cs));
        MF3D_CK(cudaStreamDestroy(bs));
        MF3D_CK(cudaGraphInstantiate(&exec_, graph_, 0));
    }

    std::vector<std::unique_ptr<HeadSolver>> hs_;
    mf3d_solver_config cfg_;
    cudaStream_t s_ = nullptr, own_stream_ = nullptr;
    bool flexible_ = false;
    int occ_[16] = {};
    int pocc_[16] = {}; // resident batched x-pair-sweep CTAs per SM, by mode
    std::vector<Op> ops_;
    std::vector<std::unique_ptr<DevMem>> retired_; // launch tables of candidates no longer used
    std::unique_ptr<DevMem> tail_mem_, pcg_mem_;
    size_t tail_smem_ = 0;
    PcgItem* items_d_ = nullptr;
    int *off3_d_ = nullptr, *off1_d_ = nullptr, *errs_d_ = nullptr, *any_d_ = nullptr;
    int tot3_ = 0, tot1_ = 0;
    CopyItem* copy_d_ = nullptr;
    PcgState* states_d_ = nullptr;
    BatchCtl* ctl_d_ = nullptr;
    CopyItem* copy_h_ = nullptr;
    PcgState* states_h_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaGraphConditionalHandle cond_ = 0;
    int pre_launches_ = 0, body_launches_ = 0, post_launches_ = 0;
};

} // namespace mf3d

// =========================================================================================
// C-ABI of the batched solves
// =========================================================================================
struct mf3d_batch {
    std::unique_ptr<BatchSolverBase> impl;
};

extern "C" {

int mf3d_batch_create(int count, const mf3d_grid* grids, const mf3d_bc* bc, const mf3d_solver_config* cfg,
                      void* stream, mf3d_batch** out) {
    return guard([&] {
        need(grids, "grids");
        need(bc, "bc");
        need(cfg, "cfg");
        need(out, "out");
        *out = nullptr;
        if (count < 1) throw Error(MF3D_E_INVALID, "count must be positive");
        for (int r = 0; r < count; ++r) check_grid(&grids[r]);
        const mf3d_solver_config c = *cfg;
        if (c.solver != MF3D_SOLVER_PCG_MG) throw Error(MF3D_E_INVALID, "batched solves support solver = PCG_MG only");
        if (c.mg_pre_smooth < 1 || c.mg_post_smooth < 1)
            throw Error(MF3D_E_INVALID, "batched solves need at least one pre- and one post-smoothing sweep");
        cudaStream_t s = (cudaStream_t)stream, own = nullptr;
        if (!s) {
            MF3D_CK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
            s = own;
        }
        try {
            std::vector<std::unique_ptr<HeadSolver>> hs;
            for (int r = 0; r < count; ++r) hs.emplace_back(new HeadSolver(grids[r], *bc, c, s));
            std::unique_ptr<mf3d_batch> b(new mf3d_batch());
            if (c.precision == MF3D_PREC_FP64)
                b->impl.reset(new BatchSolverT<double, double>(std::move(hs), c, s, own));
            else if (c.precision == MF3D_PREC_FP32)
                b->impl.reset(new BatchSolverT<float, float>(std::move(hs), c, s, own));
            else if (c.precision == MF3D_PREC_BF16)
                b->impl.reset(new BatchSolverT<float, __nv_bfloat16>(std::move(hs), c, s, own));
            else
                throw Error(MF3D_E_INVALID, "unknown precision");
            *out = b.release();
        } catch (...) {
            if (own) {
                cudaStreamSynchronize(own);
                cudaStreamDestroy(own);
            }
            throw;
        }
    });
}

int mf3d_batch_destroy(mf3d_batch* b) {
    return guard([&] { delete b; });
}

int mf3d_batch_count(const mf3d_batch* b) { return b ? b->impl->count() : -1; }

long long mf3d_batch_device_bytes(const mf3d_batch* b) { return b ? b->impl->device_bytes() : -1; }

int mf3d_batch_set_K(mf3d_batch* b, const double* const* K) {
    return guard([&] {
        need(b, "batch");
        need(K, "K");
        for (int r = 0; r < b->impl->count(); ++r) need(K[r], "K[r]");
        b->impl->set_K(K);
    });
}

int mf3d_batch_solve(mf3d_batch* b, double* const* h, const double* const* x0, mf3d_solve_result* res) {
    return guard([&] {
        need(b, "batch");
        need(h, "h");
        b->impl->solve(h, x0, res);
    });
}

int mf3d_batch_autotune(mf3d_batch* b, int reps, mf3d_batch_tuning* out, int cap, int* count) {
    return guard([&] {
        need(b, "batch");
        const std::vector<mf3d_batch_tuning> t = b->impl->autotune(reps);
        const int n = std::min<int>((int)t.size(), std::max(0, cap));
        for (int i = 0; i < n && out; ++i) out[i] = t[i];
        if (count) *count = (int)t.size();
    });
}

} // extern "C"
