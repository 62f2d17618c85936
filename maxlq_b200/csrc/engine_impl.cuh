// engine_impl.cuh -- pipelines and programs of Engine<T> (see engine.cuh);
// instantiated once per precision by engine_f32.cu and engine_f64.cu.
#pragma once
#include "engine_common.cuh"

namespace mlq {

// ----------------------------------------------------------------------------
// Engine<T>: buffers
// ----------------------------------------------------------------------------
template <typename T>
Engine<T>::Engine(const mlq_params& p) : EngineBase(p) {
    nxcap = b2.nx;
    nbcap = b2.nb;
    // bands of fractional dealias orders reached by the |u|^k chains
    auto widen = [&](double k) {
        while (k + MACH_EPSILON >= 2.0) k -= 2.0;
        if (k > 1.0) {
            const Band b = make_band(band_cut_for_order(n, k));
            nxcap = std::max(nxcap, b.nx);
            nbcap = std::max(nbcap, b.nb);
        }
    };
    widen(P.q - 2.0);
    widen(P.q / 2.0);
    if (!use_e_u) widen(P.q - 4.0);
    reg_ok_ = n >= 64 && (n & (n - 1)) == 0;
    cfft_ok_ = reg_ok_ && n <= 1024;
    if (const char* kv = std::getenv("MLQ_PASS_KERNELS")) cfft_ok_ = cfft_ok_ && std::string(kv) != "reg";
    pitch_even_ = cfft_ok_ && sizeof(T) == 4;
    // the mixed path keeps its CG state (every state vector's Fourier
    // coefficients) in FP32; the operations on it compute in FP64
    state32_ = sizeof(T) == 4;
    if (const char* e = std::getenv("MLQ_STATE_F64")) state32_ = state32_ && std::string(e) != "1";
    if (const char* e = std::getenv("MLQ_DEVICE_LS")) ls_dev_on_ = std::string(e) != "0";
    if (const char* e = std::getenv("MLQ_LS_TRANSFORM_TRIALS")) ls_transform_trials_ = std::string(e) == "1";
    {
        int dev = 0;
        MLQ_CUDA(cudaGetDevice(&dev));
        MLQ_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
    }
    ereg_ = (n > 512 && sizeof(T) == 4) ? 16 : 8;
    long ntw = 0;
    for (const auto& kv : tw_off) ntw = std::max<long>(ntw, kv.second + kv.first);
    if (sizeof(T) == 8) {
        d_twT_ = reinterpret_cast<cpx<T>*>(d_tw);
    } else {
        d_twT_ = (cpx<T>*)dev_alloc(ntw * sizeof(cpx<T>));
        std::vector<cpx<double>> h(ntw);
        MLQ_CUDA(cudaMemcpyAsync(h.data(), d_tw, ntw * sizeof(cpx<double>), cudaMemcpyDeviceToHost, stream));
        MLQ_CUDA(cudaStreamSynchronize(stream));
        std::vector<cpx<T>> hf(ntw);
        for (long i = 0; i < ntw; ++i) hf[i] = mk<T>((T)h[i].x, (T)h[i].y);
        MLQ_CUDA(cudaMemcpyAsync(d_twT_, hf.data(), ntw * sizeof(cpx<T>), cudaMemcpyHostToDevice, stream));
        MLQ_CUDA(cudaStreamSynchronize(stream));
    }
    tune_yz();
    // z-slab streaming when the physical fields the programs keep resident
    // (up to ~72 with the line-search setup) would not fit in free memory;
    // MLQ_SLAB_PLANES=k forces k planes per slab (0: never)
    if (cfft_ok_) {
        int want = -1;
        if (const char* e = std::getenv("MLQ_SLAB_PLANES")) {
            want = std::atoi(e) > 0 ? std::atoi(e) : -1;
        } else {
            size_t fr = 0, tot = 0;
            MLQ_CUDA(cudaMemGetInfo(&fr, &tot));
            if (72.0 * (double)n3 * sizeof(T) > 0.6 * (double)fr) want = 0;
        }
        if (want >= 0) {
            int zs = 1;
            if (want > 0) {
                while (zs * 2 <= want && zs * 2 <= n) zs *= 2;
            } else {
                // about 4 GB of slab buffers for up to 24 distinct inputs
                while (zs * 2 <= n && 24.0 * (zs * 2) * (double)n * n * sizeof(T) <= 4.0e9) zs *= 2;
            }
            slab_ = true;
            zs_ = zs;
            graphs_on_ = false;  // slot storage moves between fields from one call to the next
        }
    }
}

template <typename T>
RPlan Engine<T>::rplan(int L) const {
    RPlan p;
    p.L = L;
    p.nst = 0;
    p.tw_off = tw_off.at(L);
    int m = L;
    for (int r : {16, 8, 4, 2}) {
        if (r > ereg_) continue;
        while (m % r == 0 && m > 1) {
            p.radix[p.nst++] = r;
            m /= r;
        }
    }
    if (m != 1) throw CudaError("register FFT needs a power-of-two length", MLQ_ERR_BADARG);
    return p;
}

// columns per y/z tile: up to 128-byte rows within a 256-thread block
template <typename T>
int Engine<T>::reg_tx() const {
    const int nT = n / ereg_;
    int tx = 128 / (int)sizeof(cpx<T>);
    while (tx > 1 && (tx * nT > 256 || (size_t)n * tx * sizeof(cpx<T>) > 96 * 1024)) tx /= 2;
    return tx;
}

// rows per x-stage block: nrows_per_line FFT rows of pitch `pitch` per line
template <typename T>
int Engine<T>::reg_lx(int nrows_per_line, size_t pitch) const {
    const int nT = (n / 2) / ereg_;
    int lx = 32;
    while (lx > 1 && (nrows_per_line * lx * nT > 256 || nrows_per_line * lx * pitch * sizeof(cpx<T>) > 96 * 1024 ||
                      ((long)n * n) % lx != 0))
        lx /= 2;
    return lx;
}

// resident blocks of a kernel on the whole device (occupancy x SMs), cached
template <typename T>
int Engine<T>::persistent_blocks(const void* kernel, int threads, size_t smem) {
    auto it = occ_.find(kernel);
    if (it != occ_.end()) return it->second;
    int nb = 0;
    MLQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem));
    if (nb < 1) throw CudaError("pass kernel does not fit on an SM", MLQ_ERR_CUDA);
    occ_[kernel] = nb * num_sms_;
    return nb * num_sms_;
}

template <typename T>
template <int NN>
void Engine<T>::xinv_c(XInvArgs<T>& xa, int narr) {
    using S = CShape<NN, T>;
    constexpr int LPB = S::XLPB;
    const size_t smem = S::XSMEM;
    auto kern = xinv_c_kernel<NN, T>;
    allow_smem(kern);
    const int G = persistent_blocks((const void*)kern, 256, smem);
    const long ng = xa.nlines / LPB;
    dim3 grid((unsigned)std::min<long>(ng, std::max(1, G / narr)), narr);
    kern<<<grid, 256, smem, stream>>>(xa, d_twT_ + tw_off.at(NN / 2), d_twT_ + tw_off.at(NN));
}

// y/z launches of tile-shape variant V (cfft.cuh YShape)
template <typename T>
template <int NN, int V>
void Engine<T>::y_cv(YArgs<T>& ya, int sign, int narr) {
    using S = YShape<NN, T, V>;
    if constexpr (S::PAIR) {
        if constexpr (std::is_same<T, float>::value) {
            using PS = PairShape<NN>;
            const size_t smem = PS::SMEM;
            const long items = (long)ya.nz * (((ya.nx + 1) / 2 + PS::NP - 1) / PS::NP);
            auto run = [&](auto kern) {
                allow_smem(kern);
                const int G = persistent_blocks((const void*)kern, PS::THREADS, smem);
                dim3 grid((unsigned)std::min<long>(items, std::max(1, G / narr)), narr);
                kern<<<grid, PS::THREADS, smem, stream>>>(ya, d_twT_ + tw_off.at(NN));
            };
            if (sign < 0)
                run(ypass_pair_kernel<NN, -1, S::PAIR_MINB>);
            else
                run(ypass_pair_kernel<NN, +1, S::PAIR_MINB>);
        }
        return;
    }
    const size_t smem = S::YSMEM;
    const long items = (long)ya.nz * ((ya.nx + S::TX - 1) / S::TX);
    auto run = [&](auto kern) {
        allow_smem(kern);
        const int G = persistent_blocks((const void*)kern, S::YTHREADS, smem);
        dim3 grid((unsigned)std::min<long>(items, std::max(1, G / narr)), narr);
        kern<<<grid, S::YTHREADS, smem, stream>>>(ya, d_twT_ + tw_off.at(NN));
    };
    if constexpr (S::CW) {
        if (sign < 0)
            run(ypass_cw_kernel<NN, V, -1, T>);
        else
            run(ypass_cw_kernel<NN, V, +1, T>);
    } else {
        if (sign < 0)
            run(ypass_c_kernel<NN, V, -1, T>);
        else
            run(ypass_c_kernel<NN, V, +1, T>);
    }
}

template <typename T>
template <int NN, int V>
void Engine<T>::zfwd_cv(ZFwdArgs<T>& za, int narr) {
    if constexpr (YShape<NN, T, V>::PAIR) {
        if constexpr (std::is_same<T, float>::value) {
            using PS = PairShape<NN>;
            const size_t smem = PS::SMEM + 2 * NN * sizeof(float);  // + the K table
            const long items = (long)za.band.nb * (((za.nx + 1) / 2 + PS::NP - 1) / PS::NP);
            auto kern = zfwd_pair_kernel<NN, YShape<NN, T, V>::PAIR_MINB>;
            allow_smem(kern);
            const int G = persistent_blocks((const void*)kern, PS::THREADS, smem);
            dim3 grid((unsigned)std::min<long>(items, std::max(1, G / narr)), narr);
            last_zblocks_ = (long)grid.x * narr;
            ensure_partials(last_zblocks_ * MAX_RED);
            za.partials = d_partials;
            kern<<<grid, PS::THREADS, smem, stream>>>(za, d_twT_ + tw_off.at(NN));
        }
        return;
    }
    using S = YShape<NN, T, V>;
    const size_t smem = S::ZSMEM;
    const long items = (long)za.band.nb * ((za.nx + S::TX - 1) / S::TX);
    auto run = [&](auto kern) {
        allow_smem(kern);
        const int G = persistent_blocks((const void*)kern, S::YTHREADS, smem);
        dim3 grid((unsigned)std::min<long>(items, std::max(1, G / narr)), narr);
        last_zblocks_ = (long)grid.x * narr;
        ensure_partials(last_zblocks_ * MAX_RED);
        za.partials = d_partials;
        kern<<<grid, S::YTHREADS, smem, stream>>>(za, d_twT_ + tw_off.at(NN));
    };
    if constexpr (S::CW)
        run(zfwd_cw_kernel<NN, V, T>);
    else
        run(zfwd_c_kernel<NN, V, T>);
}

template <typename T>
template <int NN, int V>
void Engine<T>::zinv_cv(ZInvArgs<T>& za, int narr) {
    if constexpr (YShape<NN, T, V>::PAIR) {
        // single-source ops run as one-output ops of the pair kernel; ops
        // that add several sources take the default tile shape
        bool single = true;
        for (int i = 0; i < narr; ++i) single = single && za.op[i].nsrc == 1;
        if (!single) {
            zinv_cv<NN, 0>(za, narr);
            return;
        }
        ZInvMultiArgs<T> zm;
        zm.n = za.n;
        zm.nx = za.nx;
        zm.band = za.band;
        zm.px = za.px;
        for (int i = 0; i < narr; ++i) {
            ZInvMultiOp& o = zm.op[i];
            o.spec = za.op[i].src[0].spec;
            o.f64 = za.op[i].src[0].f64;
            o.nout = 1;
            o.sym[0] = za.op[i].src[0].sym;
            o.ab[0] = za.op[i].src[0].ab;
            o.coef[0] = za.op[i].src[0].coef;
            o.ys_out[0] = za.op[i].ys_out;
        }
        zinv_multi_cv<NN, V>(zm, narr);
        return;
    }
    using S = YShape<NN, T, V>;
    const size_t smem = S::ZISMEM;
    const long items = (long)za.band.nb * ((za.nx + S::TX - 1) / S::TX);
    auto run = [&](auto kern) {
        allow_smem(kern);
        const int G = persistent_blocks((const void*)kern, S::YTHREADS, smem);
        dim3 grid((unsigned)std::min<long>(items, std::max(1, G / narr)), narr);
        kern<<<grid, S::YTHREADS, smem, stream>>>(za, d_twT_ + tw_off.at(NN));
    };
    if constexpr (S::CW)
        run(zinv_cw_kernel<NN, V, T>);
    else
        run(zinv_c_kernel<NN, V, T>);
}

// f(std::integral_constant<int, V>) for the variant chosen for pass `kind`
template <typename T>
template <int NN, class Fn>
void Engine<T>::with_variant(int kind, Fn&& f) {
    const int v = yvar_[kind];
    if constexpr (YShape<NN, T, 1>::valid) {
        if (v == 1) return f(std::integral_constant<int, 1>{});
    }
    if constexpr (YShape<NN, T, 2>::valid) {
        if (v == 2) return f(std::integral_constant<int, 2>{});
    }
    if constexpr (YShape<NN, T, 3>::valid) {
        if (v == 3) return f(std::integral_constant<int, 3>{});
    }
    if constexpr (YShape<NN, T, 4>::valid) {
        if (v == 4) return f(std::integral_constant<int, 4>{});
    }
    if constexpr (YShape<NN, T, 5>::valid) {
        if (v == 5) return f(std::integral_constant<int, 5>{});
    }
    if constexpr (YShape<NN, T, 6>::valid) {
        if (v == 6) return f(std::integral_constant<int, 6>{});
    }
    if constexpr (YShape<NN, T, 7>::valid) {
        if (v == 7) return f(std::integral_constant<int, 7>{});
    }
    if constexpr (YShape<NN, T, 8>::valid) {
        if (v == 8) return f(std::integral_constant<int, 8>{});
    }
    if constexpr (YShape<NN, T, 9>::valid) {
        if (v == 9) return f(std::integral_constant<int, 9>{});
    }
    f(std::integral_constant<int, 0>{});
}

template <typename T>
template <int NN>
void Engine<T>::y_c(YArgs<T>& ya, int sign, int narr) {
    with_variant<NN>(sign < 0 ? YV_YFWD : YV_YINV,
                     [&](auto vc) { this->template y_cv<NN, decltype(vc)::value>(ya, sign, narr); });
}

template <typename T>
template <int NN>
void Engine<T>::zfwd_c(ZFwdArgs<T>& za, int narr) {
    bool rt = false;
    for (int i = 0; i < narr; ++i) rt = rt || za.op[i].ys_out != nullptr;
    with_variant<NN>(rt ? YV_ZRT : YV_ZFWD,
                     [&](auto vc) { this->template zfwd_cv<NN, decltype(vc)::value>(za, narr); });
}

template <typename T>
template <int NN>
void Engine<T>::zinv_c(ZInvArgs<T>& za, int narr) {
    with_variant<NN>(YV_ZINV, [&](auto vc) { this->template zinv_cv<NN, decltype(vc)::value>(za, narr); });
}

template <typename T>
std::string Engine<T>::kernel_config() const {
    const char* fam = cfft_ok_ ? "compile-time" : (reg_ok_ ? "register" : "shared-memory");
    std::string r = std::string("{\"precision\": \"") + (sizeof(T) == 4 ? "fp32" : "fp64") +
                    "\", \"pass_kernels\": \"" + fam + "\", \"slab_planes\": " + std::to_string(slab_ ? zs_ : 0) +
                    ", \"graph_replays\": " + std::to_string(graph_launches_) +
                    ", \"line_search_trials_polynomial\": " + std::to_string(ls_poly_trials_) +
                    ", \"line_search_trials_transform\": " + std::to_string(ls_fft_trials_) +
                    ", \"line_searches_on_device\": " + std::to_string(ls_dev_searches_) +
                    ", \"line_search_device_passes\": " + std::to_string(ls_dev_loops_) +
                    ", \"device_bytes_peak\": " + std::to_string(bytes_peak) +
                    ", \"yz_variants\": \"" + (tune_report_.empty() ? std::string("default") : tune_report_) + "\"}";
    return r;
}

// Autotuner: time every valid y/z tile-shape variant of each pass kind on
// scratch buffers of the state band (three arrays, as the programs launch
// them) and keep the fastest.  Runs once per engine, before the programs
// allocate their buffers.  MLQ_AUTOTUNE=0 keeps variant 0 everywhere.
template <typename T>
void Engine<T>::tune_yz() {
    tune_report_.clear();
    if (!cfft_ok_) return;
    if (const char* e = std::getenv("MLQ_AUTOTUNE"))
        if (std::string(e) == "0") return;
    bool any = false;
    dispatch_n(n, [&](auto nc) {
        constexpr int NN = decltype(nc)::value;
        any = YShape<NN, T, 1>::valid || YShape<NN, T, 2>::valid || YShape<NN, T, 3>::valid || YShape<NN, T, 8>::valid ||
              YShape<NN, T, 5>::valid || YShape<NN, T, 6>::valid || YShape<NN, T, 7>::valid;
    });
    if (!any) return;
    if (const char* e = std::getenv("MLQ_YZ_VARIANTS")) {  // one fixed variant per pass kind (measurement runs)
        std::vector<int> v;
        for (const char* c = e; *c;) {
            v.push_back(std::atoi(c));
            while (*c && *c != ',') ++c;
            if (*c == ',') ++c;
        }
        bool ok = (int)v.size() == YV_KINDS;
        for (int k = 0; ok && k < YV_KINDS; ++k)
            dispatch_n(n, [&](auto nc) {
                constexpr int NN = decltype(nc)::value;
                const int x = v[k];
                ok = ok && (x == 0 || (x == 1 && YShape<NN, T, 1>::valid) || (x == 2 && YShape<NN, T, 2>::valid) ||
                            (x == 3 && YShape<NN, T, 3>::valid) || (x == 4 && YShape<NN, T, 4>::valid) ||
                            (x == 5 && YShape<NN, T, 5>::valid) || (x == 6 && YShape<NN, T, 6>::valid) ||
                            (x == 7 && YShape<NN, T, 7>::valid) || (x == 8 && YShape<NN, T, 8>::valid) ||
                            (x == 9 && YShape<NN, T, 9>::valid));
            });
        if (ok) {
            for (int k = 0; k < YV_KINDS; ++k) yvar_[k] = v[k];
            tune_report_ = std::string("fixed by MLQ_YZ_VARIANTS=") + e;
            return;
        }
    }
    if (const char* e = std::getenv("MLQ_YZ_VARIANT")) {  // fixed variant (measurement runs)
        const int v = std::atoi(e);
        bool ok = v == 0;
        dispatch_n(n, [&](auto nc) {
            constexpr int NN = decltype(nc)::value;
            ok = ok || (v == 1 && YShape<NN, T, 1>::valid) || (v == 2 && YShape<NN, T, 2>::valid) ||
                 (v == 3 && YShape<NN, T, 3>::valid) || (v == 4 && YShape<NN, T, 4>::valid) ||
                 (v == 5 && YShape<NN, T, 5>::valid) || (v == 6 && YShape<NN, T, 6>::valid) ||
                 (v == 7 && YShape<NN, T, 7>::valid) || (v == 8 && YShape<NN, T, 8>::valid) ||
                 (v == 9 && YShape<NN, T, 9>::valid);
        });
        if (ok)
            for (int k = 0; k < YV_KINDS; ++k) yvar_[k] = v;
        tune_report_ = std::string("fixed by MLQ_YZ_VARIANT=") + e;
        return;
    }
    const Band b = b2;
    constexpr int NA = 3;
    const int pxb = px_of(b);
    const long xs_n = (long)n * n * pxb, ys_n = (long)n * b.nb * pxb, sp_n = (long)b.nb * b.nb * b.nx;
    cpx<T>* A = (cpx<T>*)dev_alloc(NA * xs_n * sizeof(cpx<T>));
    cpx<T>* B = (cpx<T>*)dev_alloc(NA * ys_n * sizeof(cpx<T>));
    // spectra in the state storage, as the programs read and write them
    char* C = (char*)dev_alloc(NA * sp_n * sv_elem());
    MLQ_CUDA(cudaMemsetAsync(A, 0, NA * xs_n * sizeof(cpx<T>), stream));
    MLQ_CUDA(cudaMemsetAsync(B, 0, NA * ys_n * sizeof(cpx<T>), stream));
    MLQ_CUDA(cudaMemsetAsync(C, 0, NA * sp_n * sv_elem(), stream));
    YArgs<T> yf{}, yi{};
    yf.n = yi.n = n;
    yf.nz = yi.nz = n;
    yf.nx = yi.nx = b.nx;
    yf.px = yi.px = pxb;
    yf.band = yi.band = b;
    ZFwdArgs<T> zf{};
    zf.n = n;
    zf.nx = b.nx;
    zf.px = pxb;
    zf.band = b;
    zf.norm = 1.0 / (double)n3;
    ZInvArgs<T> zi{};
    zi.n = n;
    zi.nx = b.nx;
    zi.px = pxb;
    zi.band = b;
    for (int a = 0; a < NA; ++a) {
        yf.in[a] = A + a * xs_n;
        yf.out[a] = B + a * ys_n;
        yi.in[a] = B + a * ys_n;
        yi.out[a] = A + a * xs_n;
        ZFwdOp op = {};
        op.in = B + a * ys_n;
        op.spec_out = C + a * sp_n * sv_elem();
        op.spec_f64 = sf64();
        op.sym = SYM_ONE;
        op.red_self = 0;
        for (int r = 0; r < 3; ++r) op.red_with_slot[r] = -1;
        zf.op[a] = op;
        ZInvOp oi = {};
        oi.src[0] = ZSrc{C + a * sp_n * sv_elem(), sf64(), SYM_IKX, 0, 1.0};
        oi.nsrc = 1;
        oi.ys_out = B + a * ys_n;
        zi.op[a] = oi;
    }
    cudaEvent_t e0, e1;
    MLQ_CUDA(cudaEventCreate(&e0));
    MLQ_CUDA(cudaEventCreate(&e1));
    const char* names[YV_KINDS] = {"y_fwd", "y_inv", "z_fwd", "z_inv", "z_roundtrip"};
    // the round-trip kind: dealias round trips in place, no spectrum, no reduction
    ZFwdArgs<T> zr = zf;
    for (int a = 0; a < NA; ++a) {
        zr.op[a].spec_out = nullptr;
        zr.op[a].red_self = -1;
        zr.op[a].ys_out = B + a * ys_n;
    }
    auto launch = [&](int kind) {
        dispatch_n(n, [&](auto nc) {
            constexpr int NN = decltype(nc)::value;
            if (kind == YV_YFWD) y_c<NN>(yf, -1, NA);
            if (kind == YV_YINV) y_c<NN>(yi, +1, NA);
            if (kind == YV_ZFWD) zfwd_c<NN>(zf, NA);
            if (kind == YV_ZINV) zinv_c<NN>(zi, NA);
            if (kind == YV_ZRT) zfwd_c<NN>(zr, NA);
        });
        MLQ_CUDA(cudaGetLastError());
    };
    constexpr int NV = 10;
    bool valid[NV] = {true, false, false, false, false, false, false, false, false, false};
    dispatch_n(n, [&](auto nc) {
        constexpr int NN = decltype(nc)::value;
        valid[1] = YShape<NN, T, 1>::valid;
        valid[2] = YShape<NN, T, 2>::valid;
        valid[3] = YShape<NN, T, 3>::valid;
        valid[4] = YShape<NN, T, 4>::valid;
        valid[5] = YShape<NN, T, 5>::valid;
        valid[6] = YShape<NN, T, 6>::valid;
        valid[7] = YShape<NN, T, 7>::valid;
        valid[8] = YShape<NN, T, 8>::valid;
        valid[9] = YShape<NN, T, 9>::valid;
    });
    auto valid_for = [&](int kind, int v) { return valid[v] && kind >= 0; };
    // every variant of every kind once first (clocks, attributes, page-in)
    for (int kind = 0; kind < YV_KINDS; ++kind)
        for (int v = 0; v < NV; ++v)
            if (valid_for(kind, v)) {
                yvar_[kind] = v;
                launch(kind);
            }
    // then round-robin single launches, best of 5 per variant; a variant
    // replaces variant 0 only when it is at least 3 % faster
    std::string rep;
    for (int kind = 0; kind < YV_KINDS; ++kind) {
        float best_ms[NV];
        std::fill(best_ms, best_ms + NV, 1e30f);
        for (int r = 0; r < 5; ++r)
            for (int v = 0; v < NV; ++v) {
                if (!valid_for(kind, v)) continue;
                yvar_[kind] = v;
                MLQ_CUDA(cudaEventRecord(e0, stream));
                launch(kind);
                MLQ_CUDA(cudaEventRecord(e1, stream));
                MLQ_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                MLQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                best_ms[v] = std::min(best_ms[v], ms);
            }
        int bestv = 0;
        std::string times;
        for (int v = 0; v < NV; ++v) {
            if (!valid_for(kind, v)) continue;
            times += (times.empty() ? "" : " ") + std::to_string(v) + ":" + std::to_string(best_ms[v]);
            if (best_ms[v] < 0.97f * best_ms[bestv]) bestv = v;
        }
        yvar_[kind] = bestv;
        rep += std::string(rep.empty() ? "" : "; ") + names[kind] + " v" + std::to_string(bestv) + " (" + times + " ms)";
    }
    MLQ_CUDA(cudaEventDestroy(e0));
    MLQ_CUDA(cudaEventDestroy(e1));
    free_dev(A);
    free_dev(B);
    free_dev(C);
    tune_report_ = rep;
}

template <typename T>
template <int NN, class F>
void Engine<T>::xfwd_c(XFwdArgs<T>& xa, const F& f) {
    using S = CShape<NN, T>;
    const size_t smem = XFwdSmem<NN, T, F::NOUT>::BYTES;
    auto kern = xfwd_c_kernel<NN, T, F>;
    allow_smem(kern);
    const int G = persistent_blocks((const void*)kern, 256, smem);
    const long ng = xa.nlines / S::XLPB;
    const int grid = (int)std::min<long>(ng, G);
    last_xblocks_ = grid;
    if (F::NRED > 0) ensure_partials((long)grid * F::NRED);
    xa.partials = d_partials;
    kern<<<grid, 256, smem, stream>>>(xa, f, d_twT_ + tw_off.at(NN / 2), d_twT_ + tw_off.at(NN));
}

template <typename T>
template <class F>
void Engine<T>::launch_xfwd(XFwdArgs<T>& xa, const F& f, int nout, const Band& b) {
    const int h = n / 2;
    xa.px = px_of(b);
    xa.nanflag = d_results + NAN_SLOT;
    // compulsory bytes: each distinct input field read once, each output written once
    int nin_distinct = 0;
    for (int i = 0; i < F::NIN; ++i) {
        bool seen = false;
        for (int j = 0; j < i; ++j) seen = seen || xa.in[j] == xa.in[i];
        nin_distinct += seen ? 0 : 1;
    }
    if (xa.nlines <= 0) xa.nlines = (long)n * n;
    const double lines = (double)xa.nlines;
    const double bytes = lines * n * sizeof(T) * nin_distinct + lines * b.nx * sizeof(cpx<T>) * nout;
    if (cfft_ok_) {
        cudaEvent_t ev = prof_mark();
        dispatch_n(n, [&](auto nc) { this->template xfwd_c<decltype(nc)::value>(xa, f); });
        launched(xfwd_name<F>(prof_detail), bytes, ev);
        return;
    }
    if (reg_ok_) {
        xa.lx = reg_lx(nout, row_pitch(h));
        xa.tw_n_off = tw_off.at(n);
        const int grid = (int)(xa.nlines / xa.lx);
        last_xblocks_ = grid;
        if (F::NRED > 0) ensure_partials((long)grid * F::NRED);
        xa.partials = d_partials;
        const size_t sm = (size_t)nout * xa.lx * row_pitch(h) * sizeof(cpx<T>);
        const int thr = nout * xa.lx * (h / ereg_);
        cudaEvent_t ev = prof_mark();
        if (ereg_ == 8) {
            allow_smem(xfwd_reg_kernel<8, T, F>);
            xfwd_reg_kernel<8, T, F><<<grid, thr, sm, stream>>>(xa, f, rplan(h), d_twT_);
        } else {
            allow_smem(xfwd_reg_kernel<16, T, F>);
            xfwd_reg_kernel<16, T, F><<<grid, thr, sm, stream>>>(xa, f, rplan(h), d_twT_);
        }
        launched(xfwd_name<F>(prof_detail), bytes, ev);
        return;
    }
    xa.lx = lx_for(nout);
    const int xgrid = (int)(xa.nlines / xa.lx);
    last_xblocks_ = xgrid;
    if (F::NRED > 0) ensure_partials((long)xgrid * F::NRED);
    xa.partials = d_partials;
    const size_t xsm = (size_t)2 * nout * xa.lx * h * sizeof(cpx<T>);
    allow_smem(xfwd_kernel<T, F>);
    cudaEvent_t ev = prof_mark();
    xfwd_kernel<T, F><<<xgrid, 256, xsm, stream>>>(xa, f);
    launched(xfwd_name<F>(prof_detail), bytes, ev);
}

template <typename T>
void Engine<T>::launch_y(YArgs<T>& ya, int sign, int narr, const Band& b) {
    ya.px = px_of(b);
    if (ya.nz <= 0) ya.nz = n;
    const double bytes = (double)narr * ya.nz * ((double)n * b.nx + (double)b.nb * b.nx) * sizeof(cpx<T>);
    const char* nm = sign < 0 ? "y_fwd" : "y_inv";
    if (cfft_ok_) {
        cudaEvent_t ev = prof_mark();
        dispatch_n(n, [&](auto nc) { this->template y_c<decltype(nc)::value>(ya, sign, narr); });
        launched(nm, bytes, ev);
        return;
    }
    if (reg_ok_) {
        const int tx = reg_tx();
        ya.tx = tx;
        const size_t sm = (size_t)n * tx * sizeof(cpx<T>);
        dim3 g((b.nx + tx - 1) / tx, ya.nz, narr);
        const int thr = tx * (n / ereg_);
        cudaEvent_t ev = prof_mark();
        if (ereg_ == 8) {
            if (sign < 0) {
                allow_smem(ypass_reg_kernel<8, -1, T>);
                ypass_reg_kernel<8, -1, T><<<g, thr, sm, stream>>>(ya, rplan(n), d_twT_);
            } else {
                allow_smem(ypass_reg_kernel<8, +1, T>);
                ypass_reg_kernel<8, +1, T><<<g, thr, sm, stream>>>(ya, rplan(n), d_twT_);
            }
        } else {
            if (sign < 0) {
                allow_smem(ypass_reg_kernel<16, -1, T>);
                ypass_reg_kernel<16, -1, T><<<g, thr, sm, stream>>>(ya, rplan(n), d_twT_);
            } else {
                allow_smem(ypass_reg_kernel<16, +1, T>);
                ypass_reg_kernel<16, +1, T><<<g, thr, sm, stream>>>(ya, rplan(n), d_twT_);
            }
        }
        launched(nm, bytes, ev);
        return;
    }
    const int tx = tx_for();
    ya.tx = tx;
    ya.plan = plan(n);
    ya.tw = d_tw;
    const size_t ysm = (size_t)2 * n * tx * sizeof(cpx<T>);
    dim3 yg((b.nx + tx - 1) / tx, ya.nz, narr);
    cudaEvent_t ev = prof_mark();
    if (sign < 0) {
        allow_smem(ypass_kernel<-1, T>);
        ypass_kernel<-1, T><<<yg, 256, ysm, stream>>>(ya);
    } else {
        allow_smem(ypass_kernel<+1, T>);
        ypass_kernel<+1, T><<<yg, 256, ysm, stream>>>(ya);
    }
    launched(nm, bytes, ev);
}

template <typename T>
void Engine<T>::launch_zfwd(ZFwdArgs<T>& za, int narr, const Band& b, bool any_rt, double zbytes) {
    za.px = px_of(b);
    if (cfft_ok_) {
        cudaEvent_t ev = prof_mark();
        dispatch_n(n, [&](auto nc) { this->template zfwd_c<decltype(nc)::value>(za, narr); });
        launched(any_rt ? "z_roundtrip" : "z_fwd", zbytes, ev);
        return;
    }
    const int tx = reg_ok_ ? reg_tx() : tx_for();
    za.tx = tx;
    dim3 zg((b.nx + tx - 1) / tx, b.nb, narr);
    const long zblocks = (long)zg.x * zg.y * zg.z;
    ensure_partials(zblocks * MAX_RED);
    za.partials = d_partials;
    if (reg_ok_) {
        const size_t sm = (size_t)n * tx * sizeof(cpx<T>);
        const int thr = tx * (n / ereg_);
        cudaEvent_t ev = prof_mark();
        if (ereg_ == 8) {
            allow_smem(zfwd_reg_kernel<8, T>);
            zfwd_reg_kernel<8, T><<<zg, thr, sm, stream>>>(za, rplan(n), d_twT_);
        } else {
            allow_smem(zfwd_reg_kernel<16, T>);
            zfwd_reg_kernel<16, T><<<zg, thr, sm, stream>>>(za, rplan(n), d_twT_);
        }
        launched(any_rt ? "z_roundtrip" : "z_fwd", zbytes, ev);
    } else {
        za.plan = plan(n);
        za.tw = d_tw;
        const size_t sm = (size_t)2 * n * tx * sizeof(cpx<T>);
        allow_smem(zfwd_kernel<T>);
        cudaEvent_t ev = prof_mark();
        zfwd_kernel<T><<<zg, 256, sm, stream>>>(za);
        launched(any_rt ? "z_roundtrip" : "z_fwd", zbytes, ev);
    }
    last_zblocks_ = zblocks;
}

template <typename T>
void Engine<T>::launch_zinv(ZInvArgs<T>& za, int narr, const Band& b, double zbytes) {
    za.px = px_of(b);
    if (cfft_ok_) {
        cudaEvent_t ev = prof_mark();
        dispatch_n(n, [&](auto nc) { this->template zinv_c<decltype(nc)::value>(za, narr); });
        launched("z_inv", zbytes, ev);
        return;
    }
    const int tx = reg_ok_ ? reg_tx() : tx_for();
    za.tx = tx;
    dim3 zg((b.nx + tx - 1) / tx, b.nb, narr);
    if (reg_ok_) {
        const size_t sm = (size_t)n * tx * sizeof(cpx<T>);
        const int thr = tx * (n / ereg_);
        cudaEvent_t ev = prof_mark();
        if (ereg_ == 8) {
            allow_smem(zinv_reg_kernel<8, T>);
            zinv_reg_kernel<8, T><<<zg, thr, sm, stream>>>(za, rplan(n), d_twT_);
        } else {
            allow_smem(zinv_reg_kernel<16, T>);
            zinv_reg_kernel<16, T><<<zg, thr, sm, stream>>>(za, rplan(n), d_twT_);
        }
        launched("z_inv", zbytes, ev);
    } else {
        za.plan = plan(n);
        za.tw = d_tw;
        const size_t sm = (size_t)2 * n * tx * sizeof(cpx<T>);
        allow_smem(zinv_kernel<T>);
        cudaEvent_t ev = prof_mark();
        zinv_kernel<T><<<zg, 256, sm, stream>>>(za);
        launched("z_inv", zbytes, ev);
    }
}

template <typename T>
template <int NN, int V>
void Engine<T>::zinv_multi_cv(ZInvMultiArgs<T>& za, int nops) {
    using S = YShape<NN, T, V>;
    if constexpr (S::PAIR) {
        if constexpr (std::is_same<T, float>::value) {
            using PS = PairShape<NN>;
            const size_t smem = (size_t)PS::TILE * sizeof(float4) + NN * sizeof(cpx<float>) + 2 * NN * sizeof(float);
            const long items = (long)za.band.nb * (((za.nx + 1) / 2 + PS::NP - 1) / PS::NP);
            auto kern = zinv_multi_pair_kernel<NN, S::PAIR_MINB>;
            allow_smem(kern);
            const int G = persistent_blocks((const void*)kern, PS::THREADS, smem);
            dim3 grid((unsigned)std::min<long>(items, std::max(1, G / nops)), nops);
            kern<<<grid, PS::THREADS, smem, stream>>>(za, d_twT_ + tw_off.at(NN));
        }
    } else if constexpr (S::CW) {  // the multi-output kernels have the plain and pair tile shapes only
        zinv_multi_cv<NN, 0>(za, nops);
    } else {
        const size_t smem = S::ZISMEM;
        const long items = (long)za.band.nb * ((za.nx + S::TX - 1) / S::TX);
        auto kern = zinv_multi_c_kernel<NN, V, T>;
        allow_smem(kern);
        const int G = persistent_blocks((const void*)kern, S::YTHREADS, smem);
        dim3 grid((unsigned)std::min<long>(items, std::max(1, G / nops)), nops);
        kern<<<grid, S::YTHREADS, smem, stream>>>(za, d_twT_ + tw_off.at(NN));
    }
}

template <typename T>
void Engine<T>::launch_zinv_multi(ZInvMultiArgs<T>& za, int nops, const Band& b, double zbytes) {
    za.px = px_of(b);
    cudaEvent_t ev = prof_mark();
    dispatch_n(n, [&](auto nc) {
        constexpr int NN = decltype(nc)::value;
        this->template with_variant<NN>(
            YV_ZINV, [&](auto vc) { this->template zinv_multi_cv<NN, decltype(vc)::value>(za, nops); });
    });
    launched("z_inv", zbytes, ev);
}

template <typename T>
void Engine<T>::launch_xinv(XInvArgs<T>& xa, int narr, const Band& b) {
    xa.px = px_of(b);
    const int h = n / 2;
    if (xa.nlines <= 0) xa.nlines = (long)n * n;
    const double bytes = (double)narr * xa.nlines * ((double)b.nx * sizeof(cpx<T>) + (double)n * sizeof(T));
    xa.tw_n_off = tw_off.at(n);
    if (cfft_ok_) {
        cudaEvent_t ev = prof_mark();
        dispatch_n(n, [&](auto nc) { this->template xinv_c<decltype(nc)::value>(xa, narr); });
        launched("x_inv", bytes, ev);
        return;
    }
    if (reg_ok_) {
        xa.lx = reg_lx(1, row_pitch(h + 1));
        const size_t sm = (size_t)xa.lx * row_pitch(h + 1) * sizeof(cpx<T>);
        dim3 xg((unsigned)(xa.nlines / xa.lx), narr);
        const int thr = xa.lx * (h / ereg_);
        cudaEvent_t ev = prof_mark();
        if (ereg_ == 8) {
            allow_smem(xinv_reg_kernel<8, T>);
            xinv_reg_kernel<8, T><<<xg, thr, sm, stream>>>(xa, rplan(h), d_twT_);
        } else {
            allow_smem(xinv_reg_kernel<16, T>);
            xinv_reg_kernel<16, T><<<xg, thr, sm, stream>>>(xa, rplan(h), d_twT_);
        }
        launched("x_inv", bytes, ev);
        return;
    }
    const size_t per = (size_t)(3 * h + 1) * sizeof(cpx<T>);
    int lx = 8;
    while (lx > 1 && (per * lx > 96 * 1024 || xa.nlines % lx != 0)) lx /= 2;
    xa.lx = lx;
    xa.plan_half = plan(h);
    xa.tw = d_tw;
    allow_smem(xinv_kernel<T>);
    dim3 xg((unsigned)(xa.nlines / lx), narr);
    cudaEvent_t ev = prof_mark();
    xinv_kernel<T><<<xg, 256, per * lx, stream>>>(xa);
    launched("x_inv", bytes, ev);
}

template <typename T>
Engine<T>::~Engine() {
    if (h_stage_) cudaFreeHost(h_stage_);
    if (xstream_) cudaStreamDestroy(xstream_);
    for (LsGraph& g : lsg_)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (h_ls_) cudaFreeHost(h_ls_);
}

template <typename T>
T* Engine<T>::phys(int i) {
    if ((int)phys_.size() <= i) phys_.resize(i + 1, nullptr);
    if (!phys_[i]) phys_[i] = (T*)dev_alloc(n3 * sizeof(T));
    return phys_[i];
}
template <typename T>
cpx<T>* Engine<T>::xsbuf(int i) {
    if ((int)xs_.size() <= i) xs_.resize(i + 1, nullptr);
    if (!xs_[i]) {
        xs_[i] = (cpx<T>*)dev_alloc((size_t)n * n * pxcap() * sizeof(cpx<T>));
        if (pitch_even_) MLQ_CUDA(cudaMemsetAsync(xs_[i], 0, (size_t)n * n * pxcap() * sizeof(cpx<T>), stream));
    }
    return xs_[i];
}
template <typename T>
cpx<T>* Engine<T>::ysbuf(int i) {
    if ((int)ys_.size() <= i) ys_.resize(i + 1, nullptr);
    if (!ys_[i]) {
        ys_[i] = (cpx<T>*)dev_alloc((size_t)n * nbcap * pxcap() * sizeof(cpx<T>));
        if (pitch_even_) MLQ_CUDA(cudaMemsetAsync(ys_[i], 0, (size_t)n * nbcap * pxcap() * sizeof(cpx<T>), stream));
    }
    return ys_[i];
}
template <typename T>
cpx<T>* Engine<T>::wspec(int i) {
    if ((int)ws_.size() <= i) ws_.resize(i + 1, nullptr);
    if (!ws_[i]) ws_[i] = (cpx<T>*)dev_alloc((size_t)spec_ncomp() * sizeof(cpx<T>));
    return ws_[i];
}

template <typename T>
void* Engine<T>::stage(size_t b) {
    if (b > h_stage_bytes_) {
        if (h_stage_) cudaFreeHost(h_stage_);
        MLQ_CUDA(cudaMallocHost((void**)&h_stage_, b));
        h_stage_bytes_ = b;
    }
    return h_stage_;
}

template <typename T>
int Engine<T>::lx_for(int nout, size_t extra) const {
    const size_t per = (size_t)2 * std::max(nout, 1) * (n / 2) * sizeof(cpx<T>) + extra;
    int lx = 8;
    while (lx > 1 && (per * lx > 96 * 1024 || ((long)n * n) % lx != 0)) lx /= 2;
    return lx;
}

template <typename T>
int Engine<T>::tx_for() const {
    int tx = 16;
    while (tx > 1 && (size_t)2 * n * tx * sizeof(cpx<T>) > 96 * 1024) tx /= 2;
    return tx;
}

// ----------------------------------------------------------------------------
// pipelines
// ----------------------------------------------------------------------------
template <typename T>
template <class F>
void Engine<T>::fwd(const Band& b, const F& f, const std::vector<int>& in, std::vector<FwdOut> outs,
                    int red_dst, int fred_dst, double norm) {
    constexpr int NOUT = F::NOUT;
    static_assert(NOUT <= MAX_ARR, "too many outputs");
    if ((int)in.size() != F::NIN || (int)outs.size() != NOUT) throw CudaError("fwd: arity", MLQ_ERR_BADARG);
    if (b.nx > nxcap || b.nb > nbcap) throw CudaError("fwd: band exceeds buffers", MLQ_ERR_BADARG);
    if (slab_) {
        fwd_slab(b, f, in, outs, red_dst, fred_dst, norm);
        return;
    }
    const int h = n / 2;
    // x stage
    XFwdArgs<T> xa;
    xa.n = n;
    xa.nx = b.nx;
    for (int i = 0; i < F::NIN; ++i) xa.in[i] = phys(in[i]);
    for (int o = 0; o < NOUT; ++o) xa.out[o] = xsbuf(o);
    xa.plan_half = plan(h);
    xa.tw_n_off = tw_off.at(n);
    xa.tw = d_tw;
    launch_xfwd(xa, f, NOUT, b);
    if (F::NRED > 0 && fred_dst >= 0) finalize((int)last_xblocks_, F::NRED, 1.0 / (double)n3, fred_dst);
    if (NOUT == 0) return;
    // y forward
    YArgs<T> ya;
    ya.n = n;
    ya.nx = b.nx;
    ya.band = b;
    for (int o = 0; o < NOUT; ++o) {
        ya.in[o] = xsbuf(o);
        ya.out[o] = ysbuf(o);
    }
    launch_y(ya, -1, NOUT, b);
    fwd_z<NOUT>(b, outs, red_dst, norm);
}

// z stage of a forward pipeline: ysbuf(o) -> spectra / reductions / round trips
template <typename T>
template <int NOUT>
void Engine<T>::fwd_z(const Band& b, const std::vector<FwdOut>& outs, int red_dst, double norm) {
    ZFwdArgs<T> za;
    za.n = n;
    za.nx = b.nx;
    za.band = b;
    bool any_rt = false;
    for (int o = 0; o < NOUT; ++o) {
        const FwdOut& fo = outs[o];
        ZFwdOp& op = za.op[o];
        op.in = ysbuf(o);
        op.spec_out = fo.spec;
        op.spec_f64 = fo.spec_f64;
        // round trip: in place (then y/x inverse), or, in slab mode, into the
        // output slot's y-stage storage
        op.ys_out = fo.phys_out < 0 ? nullptr : (slab_ ? (void*)slot_ys(fo.phys_out) : (void*)ysbuf(o));
        any_rt |= fo.phys_out >= 0;
        op.sym = fo.sym;
        op.sym_ab = fo.ab;
        op.add = fo.add;
        op.add_f64 = fo.add_f64;
        op.add_sym = fo.add_sym;
        op.add_ab = fo.add_ab;
        op.add_coef = fo.add_coef;
        op.red_self = fo.red_self;
        for (int r = 0; r < 3; ++r) {
            op.red_with[r] = fo.red_with[r];
            op.red_with_f64[r] = fo.red_with_f64[r];
            op.red_with_slot[r] = fo.red_with_slot[r];
        }
    }
    za.norm = norm > 0 ? norm : 1.0 / (double)n3;
    double zbytes = 0;
    {
        const double ys_b = (double)n * b.nb * b.nx * sizeof(cpx<T>);
        const double sp_elems = (double)b.nb * b.nb * b.nx;
        for (int o = 0; o < NOUT; ++o) {
            const FwdOut& fo = outs[o];
            zbytes += ys_b;
            if (fo.spec) zbytes += sp_elems * (fo.spec_f64 ? 16 : 8);
            if (fo.phys_out >= 0) zbytes += ys_b;
            if (fo.add) zbytes += sp_elems * (fo.add_f64 ? 16 : 8);
            for (int r = 0; r < 3; ++r)
                if (fo.red_with[r]) zbytes += sp_elems * (fo.red_with_f64[r] ? 16 : 8);
        }
    }
    launch_zfwd(za, NOUT, b, any_rt, zbytes);
    const long zblocks = last_zblocks_;
    if (red_dst >= 0) finalize((int)zblocks, MAX_RED, 1.0, red_dst);
    if (slab_) {
        for (int o = 0; o < NOUT; ++o)
            if (outs[o].phys_out >= 0) {
                PSlot& sl = slot(outs[o].phys_out);
                sl.kind = PSlot::YS;
                sl.band = b;
            }
        return;
    }
    if (any_rt) {
        std::vector<cpx<T>*> ys;
        std::vector<int> po;
        for (int o = 0; o < NOUT; ++o)
            if (outs[o].phys_out >= 0) {
                ys.push_back(ysbuf(o));
                po.push_back(outs[o].phys_out);
            }
        yx_inverse(b, ys, po);
    }
}

template <typename T>
void Engine<T>::yx_inverse(const Band& b, const std::vector<cpx<T>*>& ys, const std::vector<int>& phys_out) {
    const int k = (int)ys.size();
    if (k == 0) return;
    // y inverse: ys[i] -> xs (xs buffers are free once the forward's y pass ran)
    YArgs<T> ya;
    ya.n = n;
    ya.nx = b.nx;
    ya.band = b;
    std::vector<cpx<T>*> xs(k);
    for (int i = 0; i < k; ++i) {
        xs[i] = xsbuf(i);
        ya.in[i] = ys[i];
        ya.out[i] = xs[i];
    }
    launch_y(ya, +1, k, b);
    // x inverse
    XInvArgs<T> xa;
    xa.n = n;
    xa.nx_in = b.nx;
    for (int i = 0; i < k; ++i) {
        xa.in[i] = xs[i];
        xa.out[i] = phys(phys_out[i]);
        phys_written(phys_out[i]);
    }
    xa.plan_half = plan(n / 2);
    xa.tw = d_tw;
    launch_xinv(xa, k, b);
}

template <typename T>
void Engine<T>::inv(const Band& b, const std::vector<InvOut>& outs) {
    if (b.nx > nxcap || b.nb > nbcap) throw CudaError("inv: band exceeds buffers", MLQ_ERR_BADARG);
    const int G = 6;
    bool multi = cfft_ok_ && multi_zinv_;
    for (const InvOut& io : outs) multi = multi && io.nsrc == 1;
    const size_t GM = multi ? MAX_ARR : G;
    for (size_t g0 = 0; g0 < outs.size(); g0 += GM) {
        const int k = (int)std::min<size_t>(GM, outs.size() - g0);
        if (multi) {
            // consecutive outputs of one source spectrum share a load
            ZInvMultiArgs<T> zm;
            zm.n = n;
            zm.nx = b.nx;
            zm.band = b;
            std::vector<cpx<T>*> ys(k);
            std::vector<int> po(k);
            int nops = 0;
            double zb = 0;
            for (int i = 0; i < k; ++i) {
                const InvOut& io = outs[g0 + i];
                ZInvMultiOp* op = nops ? &zm.op[nops - 1] : nullptr;
                if (!op || op->nout == ZMULTI || op->spec != io.src[0].spec || op->f64 != io.src[0].f64) {
                    op = &zm.op[nops++];
                    op->spec = io.src[0].spec;
                    op->f64 = io.src[0].f64;
                    op->nout = 0;
                    zb += (double)b.nb * b.nb * b.nx * (io.src[0].f64 ? 16 : 8);
                }
                const int o = op->nout++;
                op->sym[o] = io.src[0].sym;
                op->ab[o] = io.src[0].ab;
                op->coef[o] = io.src[0].coef;
                ys[i] = slab_ ? slot_ys(io.phys_out) : ysbuf(i);
                op->ys_out[o] = ys[i];
                po[i] = io.phys_out;
                zb += (double)n * b.nb * b.nx * sizeof(cpx<T>);
            }
            launch_zinv_multi(zm, nops, b, zb);
            if (slab_) {
                for (int i = 0; i < k; ++i) {
                    PSlot& sl = slot(po[i]);
                    sl.kind = PSlot::YS;
                    sl.band = b;
                }
                continue;
            }
            yx_inverse(b, ys, po);
            continue;
        }
        ZInvArgs<T> za;
        za.n = n;
        za.nx = b.nx;
        za.band = b;
        std::vector<cpx<T>*> ys(k);
        std::vector<int> po(k);
        for (int i = 0; i < k; ++i) {
            const InvOut& io = outs[g0 + i];
            ZInvOp& op = za.op[i];
            for (int s = 0; s < 3; ++s) op.src[s] = io.src[s];
            op.nsrc = io.nsrc;
            ys[i] = slab_ ? slot_ys(io.phys_out) : ysbuf(i);
            op.ys_out = ys[i];
            po[i] = io.phys_out;
        }
        double zb = 0;
        for (int i = 0; i < k; ++i) {
            const InvOut& io = outs[g0 + i];
            zb += (double)n * b.nb * b.nx * sizeof(cpx<T>);
            for (int s2 = 0; s2 < io.nsrc; ++s2) zb += (double)b.nb * b.nb * b.nx * (io.src[s2].f64 ? 16 : 8);
        }
        launch_zinv(za, k, b, zb);
        if (slab_) {
            for (int i = 0; i < k; ++i) {
                PSlot& sl = slot(po[i]);
                sl.kind = PSlot::YS;
                sl.band = b;
            }
            continue;
        }
        yx_inverse(b, ys, po);
    }
}

template <typename T>
__global__ void fill_kernel(T* p, long cnt, T v) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (long)gridDim.x * blockDim.x) p[i] = v;
}

template <typename T>
template <class F>
void Engine<T>::pointwise(const F& f, const std::vector<int>& in, const std::vector<int>& out, int fred_dst) {
    static_assert(F::NIN <= PArgs<T>::MAX_IN && F::NOUT <= PArgs<T>::MAX_OUT, "pointwise arity");
    if ((int)in.size() != F::NIN || (int)out.size() != F::NOUT)
        throw CudaError("pointwise: argument count does not match the functor", MLQ_ERR_BADARG);
    if (slab_) {
        if constexpr (F::NOUT > 0) {
            // the only pointwise outputs are the |u|^k powers of the calc_uk
            // chain: kept as a recipe, evaluated per slab where they are read
            if constexpr (std::is_same<F, FGPow>::value) {
                PSlot& o = slot(out[0]);
                o.kind = PSlot::RAW;
                o.src = in[0];
                o.pk = f.k;
                o.pthresh = f.thresh;
                return;
            } else {
                throw CudaError("pointwise outputs are not kept in slab mode", MLQ_ERR_BADARG);
            }
        }
        std::vector<int> uniq, which(F::NIN);
        for (int i = 0; i < F::NIN; ++i) {
            const auto it = std::find(uniq.begin(), uniq.end(), in[i]);
            which[i] = (int)(it - uniq.begin());
            if (it == uniq.end()) uniq.push_back(in[i]);
        }
        PArgs<T> a;
        a.npts = (long)zs_ * n * n;
        const int grid = grid_for(a.npts, RED_THREADS, 148 * 8);
        for (int z0 = 0; z0 < n; z0 += zs_) {
            const std::vector<const T*> ptr = expand_many(uniq, z0);
            for (int i = 0; i < F::NIN; ++i) a.in[i] = ptr[which[i]];
            ensure_partials((long)grid * std::max(F::NRED, 1));
            a.partials = d_partials;
            cudaEvent_t ev = prof_mark();
            pointwise_kernel<T, F><<<grid, RED_THREADS, 0, stream>>>(a, f);
            launched("pointwise", (double)a.npts * sizeof(T) * (F::NIN + F::NOUT), ev);
            if (F::NRED > 0 && fred_dst >= 0) finalize(grid, F::NRED, 1.0 / (double)n3, fred_dst, z0 > 0);
        }
        return;
    }
    PArgs<T> a;
    a.npts = n3;
    for (int i = 0; i < F::NIN; ++i) a.in[i] = phys(in[i]);
    for (int o = 0; o < F::NOUT; ++o) {
        a.out[o] = phys(out[o]);
        phys_written(out[o]);
    }
    const int grid = grid_for(n3, RED_THREADS, 148 * 8);
    ensure_partials((long)grid * std::max(F::NRED, 1));
    a.partials = d_partials;
    cudaEvent_t ev = prof_mark();
    pointwise_kernel<T, F><<<grid, RED_THREADS, 0, stream>>>(a, f);
    launched("pointwise", (double)n3 * sizeof(T) * (F::NIN + F::NOUT), ev);
    if (F::NRED > 0 && fred_dst >= 0) finalize(grid, F::NRED, 1.0 / (double)n3, fred_dst);
}

// ---- slab mode -------------------------------------------------------------
template <typename T>
typename Engine<T>::PSlot& Engine<T>::slot(int i) {
    if ((int)slot_.size() <= i) slot_.resize(i + 1);
    return slot_[i];
}

template <typename T>
cpx<T>* Engine<T>::slot_ys(int i) {
    if ((int)slot_ys_.size() <= i) slot_ys_.resize(i + 1, nullptr);
    if (!slot_ys_[i]) {
        if (!slot_pool_.empty()) {
            slot_ys_[i] = slot_pool_.back();
            slot_pool_.pop_back();
        } else {
            slot_ys_[i] = (cpx<T>*)dev_alloc((size_t)n * nbcap * pxcap() * sizeof(cpx<T>));
            if (pitch_even_)
                MLQ_CUDA(cudaMemsetAsync(slot_ys_[i], 0, (size_t)n * nbcap * pxcap() * sizeof(cpx<T>), stream));
        }
    }
    return slot_ys_[i];
}

template <typename T>
void Engine<T>::release_slots(int lo, int hi) {
    for (int i = lo; i < hi && i < (int)slot_ys_.size(); ++i)
        if (slot_ys_[i]) {
            slot_pool_.push_back(slot_ys_[i]);
            slot_ys_[i] = nullptr;
        }
    for (int i = lo; i < hi && i < (int)slot_.size(); ++i)
        if (slot_[i].kind != PSlot::FULL) slot_[i] = PSlot{};
}

template <typename T>
std::vector<const T*> Engine<T>::expand_many(const std::vector<int>& in, int z0) {
    std::vector<const T*> ptr(in.size(), nullptr);
    std::vector<int> batch;  // y-stage slots waiting for a shared launch
    Band bb{};
    auto flush = [&]() {
        if (batch.empty()) return;
        YArgs<T> ya{};
        ya.n = n;
        ya.nx = bb.nx;
        ya.band = bb;
        ya.nz = zs_;
        XInvArgs<T> xa{};
        xa.n = n;
        xa.nx_in = bb.nx;
        xa.nlines = (long)zs_ * n;
        xa.plan_half = plan(n / 2);
        xa.tw = d_tw;
        for (size_t j = 0; j < batch.size(); ++j) {
            ya.in[j] = slot_ys_[in[batch[j]]] + (long)z0 * bb.nb * px_of(bb);
            ya.out[j] = xslab(MAX_ARR + (int)j);
            xa.in[j] = xslab(MAX_ARR + (int)j);
            xa.out[j] = slab_buf(batch[j]);
        }
        launch_y(ya, +1, (int)batch.size(), bb);
        launch_xinv(xa, (int)batch.size(), bb);
        for (int k : batch) ptr[k] = slab_buf(k);
        batch.clear();
    };
    for (size_t k = 0; k < in.size(); ++k) {
        const PSlot& s = slot(in[k]);
        if (s.kind != PSlot::YS) continue;
        if (!batch.empty() && (s.band.cut != bb.cut || (int)batch.size() == MAX_ARR)) flush();
        bb = s.band;
        batch.push_back((int)k);
    }
    flush();
    for (size_t k = 0; k < in.size(); ++k)
        if (!ptr[k]) ptr[k] = expand(in[k], z0, (int)k);
    return ptr;
}

// the line-search setup holds 39 y-stage slots; program slots (0..59) are
// released first, so it needs 39 blocks minus what the pool already holds
template <typename T>
bool Engine<T>::ls_fits() {
    if (!slab_) return true;
    size_t fr = 0, tot = 0;
    MLQ_CUDA(cudaMemGetInfo(&fr, &tot));
    long held = (long)slot_pool_.size();
    for (int i = 0; i < 60 && i < (int)slot_ys_.size(); ++i) held += slot_ys_[i] ? 1 : 0;
    for (int i = 60; i < (int)slot_ys_.size(); ++i) held += slot_ys_[i] ? 1 : 0;
    const double blk = (double)n * nbcap * pxcap() * sizeof(cpx<T>);
    return (39.0 - (double)held) * blk < 0.9 * (double)fr;
}

template <typename T>
T* Engine<T>::slab_buf(int k) {
    if ((int)slab_bufs_.size() <= k) slab_bufs_.resize(k + 1, nullptr);
    if (!slab_bufs_[k]) slab_bufs_[k] = (T*)dev_alloc((size_t)zs_ * n * n * sizeof(T));
    return slab_bufs_[k];
}

template <typename T>
cpx<T>* Engine<T>::xslab(int k) {
    if ((int)xslab_.size() <= k) xslab_.resize(k + 1, nullptr);
    if (!xslab_[k]) {
        xslab_[k] = (cpx<T>*)dev_alloc((size_t)zs_ * n * pxcap() * sizeof(cpx<T>));
        if (pitch_even_) MLQ_CUDA(cudaMemsetAsync(xslab_[k], 0, (size_t)zs_ * n * pxcap() * sizeof(cpx<T>), stream));
    }
    return xslab_[k];
}

template <typename T>
const T* Engine<T>::expand(int i, int z0, int k) {
    const PSlot s = slot(i);
    const long npts = (long)zs_ * n * n;
    switch (s.kind) {
        case PSlot::FULL: return phys_[i] + (long)z0 * n * n;
        case PSlot::ONE: {
            T* d = slab_buf(k);
            fill_kernel<T><<<grid_for(npts, 256), 256, 0, stream>>>(d, npts, T(1));
            launched();
            return d;
        }
        case PSlot::YS: {
            // y inverse of the slab's planes, then the x inverse (c2r)
            YArgs<T> ya{};
            ya.n = n;
            ya.nx = s.band.nx;
            ya.band = s.band;
            ya.nz = zs_;
            ya.in[0] = slot_ys_[i] + (long)z0 * s.band.nb * px_of(s.band);
            ya.out[0] = xslab(MAX_ARR);
            launch_y(ya, +1, 1, s.band);
            XInvArgs<T> xa{};
            xa.n = n;
            xa.nx_in = s.band.nx;
            xa.nlines = (long)zs_ * n;
            xa.in[0] = xslab(MAX_ARR);
            xa.out[0] = slab_buf(k);
            xa.plan_half = plan(n / 2);
            xa.tw = d_tw;
            launch_xinv(xa, 1, s.band);
            return slab_buf(k);
        }
        case PSlot::RAW: {
            const T* src = expand(s.src, z0, k);
            FGPow fp;
            fp.k = s.pk;
            fp.thresh = s.pthresh;
            PArgs<T> a;
            a.npts = npts;
            a.in[0] = src;
            a.out[0] = slab_buf(k);
            const int grid = grid_for(npts, RED_THREADS, 148 * 8);
            a.partials = d_partials;
            cudaEvent_t ev = prof_mark();
            pointwise_kernel<T, FGPow><<<grid, RED_THREADS, 0, stream>>>(a, fp);
            launched("pointwise", (double)npts * sizeof(T) * 2, ev);
            return slab_buf(k);
        }
        default: break;
    }
    throw CudaError("physical field " + std::to_string(i) + " has no values", MLQ_ERR_CUDA);
}

template <typename T>
template <class F>
void Engine<T>::fwd_slab(const Band& b, const F& f, const std::vector<int>& in, std::vector<FwdOut>& outs,
                         int red_dst, int fred_dst, double norm) {
    constexpr int NOUT = F::NOUT;
    std::vector<int> uniq, which(F::NIN);
    for (int i = 0; i < F::NIN; ++i) {
        const auto it = std::find(uniq.begin(), uniq.end(), in[i]);
        which[i] = (int)(it - uniq.begin());
        if (it == uniq.end()) uniq.push_back(in[i]);
    }
    XFwdArgs<T> xa{};
    xa.n = n;
    xa.nx = b.nx;
    xa.nlines = (long)zs_ * n;
    xa.plan_half = plan(n / 2);
    xa.tw_n_off = tw_off.at(n);
    xa.tw = d_tw;
    for (int o = 0; o < NOUT; ++o) xa.out[o] = xslab(o);
    YArgs<T> ya{};
    ya.n = n;
    ya.nx = b.nx;
    ya.band = b;
    ya.nz = zs_;
    for (int z0 = 0; z0 < n; z0 += zs_) {
        const std::vector<const T*> ptr = expand_many(uniq, z0);
        for (int i = 0; i < F::NIN; ++i) xa.in[i] = ptr[which[i]];
        launch_xfwd(xa, f, NOUT, b);
        if (F::NRED > 0 && fred_dst >= 0) finalize((int)last_xblocks_, F::NRED, 1.0 / (double)n3, fred_dst, z0 > 0);
        if constexpr (NOUT > 0) {
            for (int o = 0; o < NOUT; ++o) {
                ya.in[o] = xslab(o);
                ya.out[o] = ysbuf(o) + (long)z0 * b.nb * px_of(b);
            }
            launch_y(ya, -1, NOUT, b);
        }
    }
    if constexpr (NOUT > 0) fwd_z<NOUT>(b, outs, red_dst, norm);
}

template <typename T>
void Engine<T>::release_io_buffers() {
    pu_of_ = nullptr;
    pm_ = PhysMemo{};
    for (auto* v : {&phys_}) {
        for (auto*& p : *v) {
            if (p) free_dev(p);
            p = nullptr;
        }
    }
    for (auto* v : {&xs_, &ys_, &ws_, &slot_ys_, &xslab_, &slot_pool_}) {
        for (auto*& p : *v) {
            if (p) free_dev(p);
            p = nullptr;
        }
    }
    slot_pool_.clear();
    for (auto*& p : slab_bufs_) {
        if (p) free_dev(p);
        p = nullptr;
    }
    slot_.clear();
}

// ----------------------------------------------------------------------------
// programs
// ----------------------------------------------------------------------------
// D = -i (K_odd . c) / |K|^2 over a band spectrum (0 at k = 0): the gradient
// of D is grad Lap^-1 div c, as SYM_KK_KSQ summed over the components
template <typename V, typename T>
__global__ void spec_div_ksq_kernel(SpecGeom g, const V* __restrict__ c0, const V* __restrict__ c1,
                                    const V* __restrict__ c2, cpx<T>* __restrict__ out) {
    const double twopi = 2.0 * 3.14159265358979311600;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < g.ncomp; i += (long)gridDim.x * blockDim.x) {
        const int fx = (int)(i % g.nx);
        const SpecRow row(g, (int)(i / g.nx));
        const double kx = twopi * (double)fx, ky = twopi * (double)row.jy, kz = twopi * (double)row.jz;
        const double ox = (2 * fx == g.n) ? 0.0 : kx;
        const double oy = (2 * band_fft_index(g.band, row.cy) == g.n) ? 0.0 : ky;
        const double oz = (2 * band_fft_index(g.band, row.cz) == g.n) ? 0.0 : kz;
        const double ksq = kx * kx + ky * ky + kz * kz;
        const double2 a = ldv(c0, i), b = ldv(c1, i), c = ldv(c2, i);
        const double vx = ox * a.x + oy * b.x + oz * c.x, vy = ox * a.y + oy * b.y + oz * c.y;
        cpx<T> r = mk(T(0), T(0));
        if (ksq != 0.0) r = mk((T)(vy / ksq), (T)(-vx / ksq));
        out[i] = r;
    }
}

namespace {
// physical scratch indices
enum : int {
    PU = 0,    // 0..2   u (or phi, w)
    PD = 3,    // 3..11  d_j u_i at 3+3i+j
    PL = 12,   // 12..14 Lap u
    PGP = 15,  // 15..17 grad p
    PS = 18,   // S = P2(|u|^2)
    PA = 19,   // A = P2(g^2)
    PV = 20,   // 20..22 V_j / E_j
    PP = 23,   // p
    PT = 24,   // aux2
    PGA = 25,  // 25..27 grad aux4
    PONES = 28,
    PCH = 29,  // 29..39 chain fields
    PIO = 40,  // host transfer scratch
    PIO2 = 41,
    PIO3 = 42,  // second host transfer buffer
};
// work spectra (band b2)
enum : int { WG2 = 0, WA = 1, WP = 2, WT = 3 /*3..5*/, WONE = 6, WCH = 7 /*7..*/ };
enum : int { WDIV = 52 };  // -i (K . c) / |K|^2 of the gradient program
}  // namespace
// line search along phi = u + tau d (q = 4): physical fields and work spectra
namespace {
enum : int {
    LU = 60,    // u (3)
    LD = 63,    // d (3)
    LDU = 66,   // d_j u_i at 66+3i+j
    LDD = 75,   // d_j d_i at 75+3i+j
    LS = 84,    // S_a = P2 coefficients of |phi|^2 (3)
    LV = 87,    // V_aj = P2 coefficients of W_j at 87+3a+j
    LP = 96,    // p_a (3)
    WLG = 40,   // work spectra: P2 coefficients of |grad phi|^2 (3)
    WLS = 43,   // work spectra: S_a (3)
    WLQ = 46,   // work spectra: -Lap^-1 P2(Q_a) (3), read by the next gradient
    WS = 49,    // work spectrum of S = P2(|u|^2) (gradient program, transport)
};
}  // namespace

// the physical-field memo covers u, grad u (0..11), S and A (18, 19) and the
// line search's u, d and their gradients (60..83)
template <typename T>
void Engine<T>::phys_written(int idx) {
    if ((idx >= PU && idx < PL) || idx == PS || idx == PA || (idx >= LU && idx < LS)) pm_ = PhysMemo{};
    if (idx == PS) ws_of_ = nullptr;
}

// S_0 of the line search is the gradient program's S when it was formed for
// the same u (field 18 and work spectrum WS), else the setup's own
template <typename T>
int Engine<T>::ls_phys(int a) const {
    return a == 0 ? ls_p0_ : LS + a;
}
template <typename T>
int Engine<T>::ls_wspec(int a) const {
    return a == 0 ? ls_w0_ : WLS + a;
}

// PU <- u + tau d from the line search's physical fields of u and d, when the
// memo holds them; records the transport fields (tr) for the next gradient
template <typename T>
bool Engine<T>::w_from_memo(const SVec* u, const SVec* d, double tau) {
    if (slab_ || !reuse_on_ || !d || !pm_.ls || pm_.u != (const void*)u || pm_.d != (const void*)d) {
        pm_ = PhysMemo{};
        return false;
    }
    const PhysMemo m = pm_;
    FAxpy3 f;
    f.tau = tau;
    pointwise(f, {m.iu, m.iu + 1, m.iu + 2, LD, LD + 1, LD + 2}, {PU, PU + 1, PU + 2});
    pm_ = m;
    pm_.ls = false;
    pm_.tr = true;
    pm_.tau = tau;
    return true;
}

template <typename T>
static constexpr int wf64() {
    return sizeof(T) == 8 ? 1 : 0;
}

// Fourier coefficients of the constant 1 in band b2: a unit k=0 mode.
template <typename T>
cpx<T>* Engine<T>::ones_spec() {
    static_assert(sizeof(cpx<T>) == 2 * sizeof(T), "layout");
    const bool fresh = (int)ws_.size() <= WONE || ws_[WONE] == nullptr;
    cpx<T>* w = wspec(WONE);
    if (fresh) {
        MLQ_CUDA(cudaMemsetAsync(w, 0, spec_ncomp() * sizeof(cpx<T>), stream));
        const cpx<T> one = mk<T>(T(1), T(0));
        MLQ_CUDA(cudaMemcpyAsync(w, &one, sizeof(cpx<T>), cudaMemcpyHostToDevice, stream));
        MLQ_CUDA(cudaStreamSynchronize(stream));
    }
    return w;
}

template <typename T>
void Engine<T>::ensure_phys(PowField& f) {
    if (f.phys >= 0) return;
    if (f.kind == PowField::ONE) {
        if (slab_) {
            slot(PONES).kind = PSlot::ONE;
            f.phys = PONES;
            return;
        }
        if ((int)phys_.size() <= PONES || phys_[PONES] == nullptr) {
            fill_kernel<T><<<grid_for(n3, 256), 256, 0, stream>>>(phys(PONES), n3, T(1));
            launched();
        }
        f.phys = PONES;
        return;
    }
    throw CudaError("power field without physical values", MLQ_ERR_CUDA);
}

// make sure a power field has a spectrum in band b2
template <typename T>
void Engine<T>::ensure_p2_spec(PowField& f) {
    if (f.spec >= 0) return;
    if (f.kind == PowField::ONE) {
        ones_spec();
        f.spec = WONE;
        return;
    }
    f.spec = WCH + 16 + spec_next_++;
    FwdOut o;
    o.spec = wspec(f.spec);
    o.spec_f64 = wf64<T>();
    fwd(b2, FCopy{}, {f.phys}, {o});
}

// S = P2(|u|^2) (calc_uk 2332-2333) must already be in phys(PS) ; computes
// A = P2(g^2), g = sqrt(max(S,0)) (2335-2339, 2309-2310): spectrum WA and,
// when asked, phys(PA).
template <typename T>
void Engine<T>::A_and_S(bool need_A_phys) {
    FwdOut oA;
    oA.spec = wspec(WA);
    oA.spec_f64 = wf64<T>();
    if (need_A_phys) oA.phys_out = PA;
    fwd(b2, FGSq{}, {PS}, {oA});
}

// calc_gk_order2 (function_ops.f90:2281-2319) on g = sqrt(max(S,0)), with
// A = P2(g^2) already computed.  Every branch produces the same field as the
// reference up to rounding: an order <= 1 dealias removes nothing, g**0 is 1,
// and P2(A*1) = A.
template <typename T>
PowField Engine<T>::chain(double k) {
    auto it = memo_.find(k);
    if (it != memo_.end()) return it->second;
    PowField f;
    f.k = k;
    if (k + MACH_EPSILON < 0.0) {
        f.kind = PowField::RAW;
        f.phys = PCH + tmp_next_++;
        FGPow fp;
        fp.k = k;
        fp.thresh = 1;
        pointwise(fp, {PS}, {f.phys});
    } else if (k + MACH_EPSILON < 2.0) {
        const int c = band_cut_for_order(n, k);
        if (c >= n / 2) {
            if (k == 0.0) {
                f.kind = PowField::ONE;
            } else {
                f.kind = PowField::RAW;
                f.phys = PCH + tmp_next_++;
                FGPow fp;
                fp.k = k;
                fp.thresh = 0;
                pointwise(fp, {PS}, {f.phys});
            }
        } else {
            const Band bk = make_band(c);
            f.kind = PowField::BAND;
            f.phys = PCH + tmp_next_++;
            FGPow fp;
            fp.k = k;
            fp.thresh = 0;
            FwdOut o;
            o.phys_out = f.phys;
            if (c == b2.cut) {
                f.spec = WCH + spec_next_++;
                o.spec = wspec(f.spec);
                o.spec_f64 = wf64<T>();
            }
            fwd(bk, fp, {PS}, {o});
        }
    } else {
        PowField prev = chain(k - 2.0);
        f.kind = PowField::BAND;
        if (prev.kind == PowField::ONE) {
            f.phys = PA;
            f.spec = WA;
        } else {
            ensure_phys(prev);
            f.phys = PCH + tmp_next_++;
            f.spec = WCH + spec_next_++;
            FwdOut o;
            o.phys_out = f.phys;
            o.spec = wspec(f.spec);
            o.spec_f64 = wf64<T>();
            fwd(b2, FMul{}, {PA, prev.phys}, {o});
        }
    }
    memo_[k] = f;
    return f;
}

// scalar Parseval dots of band-b2 work spectra
template <typename T>
struct SDotArgs {
    SpecGeom g;
    const cpx<T>* a[6];
    const cpx<T>* b[6];
    int np;
    double* partials;
};

template <typename T>
__global__ void __launch_bounds__(RED_THREADS) spec_sdot_kernel(SDotArgs<T> a) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.g.ncomp; i += (long)gridDim.x * blockDim.x) {
        const int fx = (int)(i % a.g.nx);
        const double w = kx_weight(a.g.n, fx);
        for (int p = 0; p < a.np; ++p) {
            const cpx<T> u = a.a[p][i], v = a.b[p][i];
            acc[p] += w * ((double)u.x * (double)v.x + (double)u.y * (double)v.y);
        }
    }
    block_reduce_store<6>(acc, a.partials, blockIdx.x);
}

template <typename T>
static void sdots(Engine<T>& e, const std::vector<std::pair<const cpx<T>*, const cpx<T>*>>& pr, int dst) {
    if (pr.size() > 6) throw CudaError("sdots: too many pairs", MLQ_ERR_BADARG);
    SDotArgs<T> a;
    a.g = e.geom(e.b2);
    a.np = (int)pr.size();
    for (int i = 0; i < a.np; ++i) {
        a.a[i] = pr[i].first;
        a.b[i] = pr[i].second;
    }
    const int grid = grid_for(a.g.ncomp, RED_THREADS, 148 * 4);
    e.ensure_partials((long)grid * 6);
    a.partials = e.d_partials;
    cudaEvent_t ev = e.prof_mark();
    spec_sdot_kernel<T><<<grid, RED_THREADS, 0, e.stream>>>(a);
    e.launched("spec_sdot", 2.0 * a.np * a.g.ncomp * sizeof(cpx<T>), ev);
    e.finalize(grid, 6, 1.0, dst);
}

// calc_local_dLqdt_inclParts (function_ops.f90:1304-1358) at phi = u + tau d,
// together with ||phi||_q^q (calc_global_Lq_norm 1675-1692).  Products are
// dealiased as the reference does; a dealias that is immediately followed by
// an L2 inner product with a band-limited field is applied through Parseval
// on the band instead of by a round trip (the projection is self-adjoint).
template <typename T>
void Engine<T>::R_eval(const SVec* u, const SVec* d, double tau, double out[3], double* lqq) {
    pu_of_ = nullptr;
    const Band& b = b2;
    const long nc = spec_ncomp();
    const double q = P.q, cv = P.visc_coef * P.visc, cp = P.press_coef;
    chain_reset();
    // 1. phi and grad phi
    std::vector<InvOut> io;
    for (int i = 0; i < 3; ++i)
        for (int j = -1; j < 3; ++j) {
            InvOut o;
            o.nsrc = d ? 2 : 1;
            const int sym = j < 0 ? SYM_ONE : SYM_IKX + j;
            o.src[0] = ZSrc{scomp(u, i), sf64(), sym, 0, 1.0};
            if (d) o.src[1] = ZSrc{scomp(d, i), sf64(), sym, 0, tau};
            o.phys_out = j < 0 ? PU + i : PD + 3 * i + j;
            io.push_back(o);
        }
    inv(b, io);
    std::vector<int> uin;
    for (int i = 0; i < 3; ++i) uin.push_back(PU + i);
    for (int i = 0; i < 9; ++i) uin.push_back(PD + i);
    // 2. first products: |u|^2 -> P2, W_j -> P2 (q>=4), grad u:grad u^T -> p,
    //    |grad u|^2 -> spectrum
    FwdOut oS, oQ, oG2;
    oS.phys_out = PS;
    oQ.sym = SYM_INV_KSQ;  // p = -Lap^-1 P2(grad u : grad u^T) (1339-1340)
    oQ.phys_out = PP;
    oG2.spec = wspec(WG2);
    oG2.spec_f64 = wf64<T>();
    if (!use_e_u) {
        FwdOut oW[3];
        for (int j = 0; j < 3; ++j) oW[j].phys_out = PV + j;
        fwd(b, FRProd{}, uin, {oS, oW[0], oW[1], oW[2], oQ, oG2});
    } else {
        fwd(b, FRProdE{}, uin, {oS, oQ, oG2});
    }
    // 3. |u|^k fields
    const bool needA = !(q == 4.0 && !use_e_u);  // for q = 4 only the spectrum of A is read
    A_and_S(needA);
    PowField a2 = chain(q - 2.0);
    PowField a4;
    if (!use_e_u) a4 = chain(q - 4.0);
    PowField ah = chain(q / 2.0);
    std::vector<std::pair<const cpx<T>*, const cpx<T>*>> pr;
    // R1 = -vc nu <a2, P2|grad u|^2>  (1318)
    ensure_p2_spec(a2);
    pr.push_back({wspec(a2.spec), wspec(WG2)});
    // ||phi||_q^q = int (|u|^{q/2})^2
    bool norm_raw = false;
    if (ah.kind == PowField::RAW) {
        norm_raw = true;
        pointwise(FSqRed{}, {ah.phys}, {}, 20);
    } else if (ah.spec < 0) {
        // a band-limited power in a wider band than P2: its full spectrum is
        // needed; integrate its square in physical space instead
        norm_raw = true;
        pointwise(FSqRed{}, {ah.phys}, {}, 20);
    } else {
        if (ah.kind == PowField::ONE) ensure_p2_spec(ah);
        pr.push_back({wspec(ah.spec), wspec(ah.spec)});
    }
    const bool direct = !use_e_u && a4.kind == PowField::ONE;
    if (direct) {
        // |u|^{q-4} = 1: R2 = -(q-2) vc nu int sum V^2, R3 = (q-2) pc int p u.V
        pointwise(FRRed1{}, {PV, PV + 1, PV + 2, PP, PU, PU + 1, PU + 2},
                  {}, 16);
    } else if (!use_e_u) {
        ensure_phys(a4);
        ensure_p2_spec(a4);
        FwdOut o[3];
        for (int i = 0; i < 3; ++i) {
            o[i].spec = wspec(WT + i);
            o[i].spec_f64 = wf64<T>();
        }
        fwd(b, FRProd2{},
            {PV, PV + 1, PV + 2, PP, PU, PU + 1, PU + 2, a4.phys},
            {o[0], o[1], o[2]});
        pr.push_back({wspec(a4.spec), wspec(WT)});
        pr.push_back({wspec(WT + 1), wspec(WT + 2)});
    } else {
        // E_j = P2(sum_i e_i d_j u_i) (calc_vgraduvgradu / calc_vvgradu, v = e_u)
        std::vector<int> ein = uin;
        ein.push_back(PS);
        FwdOut oE[3];
        for (int j = 0; j < 3; ++j) oE[j].phys_out = PV + j;
        fwd(b, FRE{}, ein, {oE[0], oE[1], oE[2]});
        ensure_phys(a2);
        FwdOut o[3];
        for (int i = 0; i < 3; ++i) {
            o[i].spec = wspec(WT + i);
            o[i].spec_f64 = wf64<T>();
        }
        fwd(b, FRProd2E{},
            {PV, PV + 1, PV + 2, PP, PU, PU + 1, PU + 2, PS,
             a2.phys},
            {o[0], o[1], o[2]});
        pr.push_back({wspec(a2.spec), wspec(WT)});
        pr.push_back({wspec(WT + 1), wspec(WT + 2)});
    }
    sdots(*this, pr, 0);
    fetch_results();
    int idx = 0;
    const double I1 = h_results[idx++];
    const double nrm = norm_raw ? h_results[20] : h_results[idx++];
    double I2, I3;
    if (direct) {
        I2 = h_results[16];
        I3 = h_results[17];
    } else {
        I2 = h_results[idx++];
        I3 = h_results[idx++];
    }
    const double R1 = -cv * I1;
    const double R2 = -cv * (q - 2.0) * I2;
    const double R3 = cp * (q - 2.0) * I3;
    out[0] = R1 + R2 + R3;
    out[1] = R1 + R2;
    out[2] = R3;
    if (lqq) *lqq = nrm;
}

// ----------------------------------------------------------------------------
// diagnostics
// ----------------------------------------------------------------------------
namespace {
enum : int { PDG2 = 100, PDR1 = 101, PDR2 = 102, PDR3 = 103, PDT1 = 104, PDT2 = 105, PDO = 106 /*106..108*/ };
}

// calc_global_dEnstrophydt: R1 = -viscCoefficient visc ||Lap u||^2 by Parseval,
// R2 = <P2((u.grad) u), Lap u> as one forward pipeline whose z stage applies
// -|K|^2 and reduces against the spectra of u (Lap is self-adjoint)
template <typename T>
void Engine<T>::dEnstrophydt(const SVec* u, double out[3]) {
    pu_of_ = nullptr;
    const long nc = spec_ncomp();
    std::vector<InvOut> io;
    for (int i = 0; i < 3; ++i)
        for (int j = -1; j < 3; ++j) {
            InvOut o;
            o.nsrc = 1;
            o.src[0] = ZSrc{scomp(u, i), sf64(), j < 0 ? SYM_ONE : SYM_IKX + j, 0, 1.0};
            o.phys_out = j < 0 ? PU + i : PD + 3 * i + j;
            io.push_back(o);
        }
    inv(b2, io);
    std::vector<int> uin;
    for (int i = 0; i < 3; ++i) uin.push_back(PU + i);
    for (int i = 0; i < 9; ++i) uin.push_back(PD + i);
    FwdOut o[3];
    for (int i = 0; i < 3; ++i) {
        o[i].sym = SYM_NEG_KSQ;
        o[i].red_with[0] = scomp(u, i);
        o[i].red_with_f64[0] = sf64();
        o[i].red_with_slot[0] = 0;
    }
    fwd(b2, FUGradU{}, uin, {o[0], o[1], o[2]}, 48);
    fetch_results();
    const double R2 = h_results[48];
    const SpecDotPair p = {u, nullptr, 4};
    double lap2 = 0.0;
    dots(&p, 1, &lap2);
    const double R1 = -P.visc_coef * P.visc * lap2;
    out[0] = R1 + R2;
    out[1] = R1;
    out[2] = R2;
}

// calc_local_pointwise_dLqdt_inclParts: the products R_eval integrates, kept
// as dealiased fields: R1 = -cv P2(a2 P2|grad u|^2), R2 = -cv (q-2) P2(a4
// P2(sum_j V_j^2)) (a2 and E_j on the e_u branch), R3 = cp (q-2) P2(P2(p a4)
// P2(u . V)) (a2, e_u . E on the e_u branch); the coefficients are applied
// after the dealias, as the reference does
template <typename T>
void Engine<T>::pointwise_R(const SVec* u, double* host) {
    if (slab_) throw CudaError("pointwise R fields need the resident (not z-slab) mode", MLQ_ERR_BADARG);
    pu_of_ = nullptr;
    const long nc = spec_ncomp();
    const double q = P.q, cv = P.visc_coef * P.visc, cp = P.press_coef;
    chain_reset();
    std::vector<InvOut> io;
    for (int i = 0; i < 3; ++i)
        for (int j = -1; j < 3; ++j) {
            InvOut o;
            o.nsrc = 1;
            o.src[0] = ZSrc{scomp(u, i), sf64(), j < 0 ? SYM_ONE : SYM_IKX + j, 0, 1.0};
            o.phys_out = j < 0 ? PU + i : PD + 3 * i + j;
            io.push_back(o);
        }
    inv(b2, io);
    std::vector<int> uin;
    for (int i = 0; i < 3; ++i) uin.push_back(PU + i);
    for (int i = 0; i < 9; ++i) uin.push_back(PD + i);
    FwdOut oS, oQ, oG2;
    oS.phys_out = PS;
    oQ.sym = SYM_INV_KSQ;  // p = -Lap^-1 P2(grad u : grad u^T) (1281-1282)
    oQ.phys_out = PP;
    oG2.phys_out = PDG2;   // P2(|grad u|^2) (calc_nablaModSquared)
    if (!use_e_u) {
        FwdOut oW[3];
        for (int j = 0; j < 3; ++j) oW[j].phys_out = PV + j;
        fwd(b2, FRProd{}, uin, {oS, oW[0], oW[1], oW[2], oQ, oG2});
    } else {
        fwd(b2, FRProdE{}, uin, {oS, oQ, oG2});
        std::vector<int> ein = uin;
        ein.push_back(PS);
        FwdOut oE[3];
        for (int j = 0; j < 3; ++j) oE[j].phys_out = PV + j;
        fwd(b2, FRE{}, ein, {oE[0], oE[1], oE[2]});
    }
    A_and_S(true);
    PowField a2 = chain(q - 2.0);
    ensure_phys(a2);
    PowField mult = a2;
    if (!use_e_u) {
        mult = chain(q - 4.0);
        ensure_phys(mult);
    }
    auto product = [&](int a, int b, int dst) {  // dst = P2(a b) (calc_uv_scalar 2069-2081)
        FwdOut o;
        o.phys_out = dst;
        fwd(b2, FMul{}, {a, b}, {o});
    };
    product(a2.phys, PDG2, PDR1);
    {
        FwdOut o;  // P2(sum_j V_j^2): calc_vgraduvgradu
        o.phys_out = PDT1;
        fwd(b2, FSq3{}, {PV, PV + 1, PV + 2}, {o});
    }
    product(mult.phys, PDT1, PDR2);
    product(PP, mult.phys, PDT2);  // P2(p |u|^{q-4}) or P2(p |u|^{q-2})
    {
        FwdOut o;  // calc_vvgradu: P2(u . V) or P2(e_u . E)
        o.phys_out = PDT1;
        if (!use_e_u)
            fwd(b2, FDot3{}, {PU, PU + 1, PU + 2, PV, PV + 1, PV + 2}, {o});
        else
            fwd(b2, FEDot{}, {PU, PU + 1, PU + 2, PS, PV, PV + 1, PV + 2}, {o});
    }
    product(PDT2, PDT1, PDR3);
    FRSum fs;
    fs.c1 = -cv;
    fs.c2 = -cv * (q - 2.0);
    fs.c3 = cp * (q - 2.0);
    pointwise(fs, {PDR1, PDR2, PDR3}, {PDO, PDO + 1, PDO + 2});
    for (int k = 0; k < 3; ++k) store_scalar_phys(PDO + k, host + k * n3);
}

// GradL2ForLq (function_ops.f90:1066-1211).  Each of the reference's five
// terms is a dealiased product; their sum is dealiased once (the projection
// is linear), the fifth term nu Lap P2(|u|^{q-2}u) is added in the spectrum.
template <typename T>
void Engine<T>::grad_l2(const SVec* u, SVec* v, SVec* c, double* lqq) {
    if (!c) throw CudaError("grad_l2 needs a spectrum buffer for |u|^{q-2}u", MLQ_ERR_BADARG);
    // u = cs w from the last line search's transport: u and grad u pointwise
    const bool rt = !slab_ && reuse_on_ && pm_.tr && pm_.next == (const void*)u;
    if (rt) {
        if (!d_coef_) d_coef_ = (double*)dev_alloc(2 * sizeof(double));
        const double h[2] = {pm_.cs, pm_.tau};
        MLQ_CUDA(cudaMemcpyAsync(d_coef_, h, sizeof(h), cudaMemcpyHostToDevice, stream));
    }
    // the same launches every CG iteration: a CUDA graph after the first two
    // (one per path: the physical fields the retraction reads are in the key)
    as_graph(rt ? (pm_.sac ? "grad_l2_rts" : "grad_l2_rt") : "grad_l2",
             {u, v, c, lqq ? (const void*)v : nullptr, rt ? (const void*)phys(pm_.idu) : nullptr},
             [&] { grad_l2_body(u, v, c, lqq != nullptr, rt); });
    pm_ = PhysMemo{};        // a replayed graph runs no host code: clear here
    if (!slab_) pu_of_ = u;  // PU, PD hold u and grad u until the next program
    ws_of_ = slab_ ? nullptr : (const void*)u;  // and PS, WS its S
    if (lqq) {
        fetch_results();
        *lqq = h_results[grad_lq_slot_];
    }
}

template <typename T>
void Engine<T>::grad_l2_body(const SVec* u, SVec* v, SVec* c, bool want_lq, bool from_retraction) {
    pu_of_ = nullptr;
    const bool sac = from_retraction && pm_.sac;
    const Band& b = b2;
    const long nc = spec_ncomp();
    const double q = P.q, cv = P.visc_coef * P.visc, cp = P.press_coef;
    chain_reset();
    // 1. u, grad u, Lap u
    std::vector<InvOut> io;
    if (from_retraction) {
        // u = cs w and grad u = cs (grad u_prev + tau grad d) from the physical
        // fields of the line search (linear in the spectra, so equal to the
        // transforms up to rounding); only Lap u is transformed
        const int idu = pm_.idu;
        pm_ = PhysMemo{};
        std::vector<int> in, out;
        for (int i = 0; i < 3; ++i) in.push_back(PU + i);
        for (int k = 0; k < 9; ++k) in.push_back(idu + k);
        for (int k = 0; k < 9; ++k) in.push_back(LDD + k);
        for (int i = 0; i < 12; ++i) out.push_back(PU + i);
        if (sac) {
            // S and A of the transport, scaled by cs^2; A's spectrum too, and
            // c = P2(A u) = cs^3 P2(A_w w) from the transport's c_tmp_
            in.push_back(PS);
            in.push_back(PA);
            out.push_back(PS);
            out.push_back(PA);
            FRetract<true> f;
            f.coef = d_coef_;
            pointwise(f, in, out);
            const long nsp = (long)b.nb * b.nb * b.nx;
            const int ws2[2] = {WA, WS};
            for (int w : ws2) {
                cudaEvent_t ew = prof_mark();
                spec_scale_pow_kernel<cpx<T>><<<grid_for(nsp, 256), 256, 0, stream>>>(wspec(w), wspec(w), nsp, d_coef_, 2);
                launched("spec_scale", 2.0 * nsp * sizeof(cpx<T>), ew);
            }
            cudaEvent_t ev = prof_mark();
            if (state32_)
                spec_scale_pow_kernel<float2><<<grid_for(3 * nc, 256), 256, 0, stream>>>(
                    (float2*)c, (const float2*)c_tmp_, 3 * nc, d_coef_, 3);
            else
                spec_scale_pow_kernel<double2><<<grid_for(3 * nc, 256), 256, 0, stream>>>(
                    (double2*)c, (const double2*)c_tmp_, 3 * nc, d_coef_, 3);
            launched("spec_scale", 2.0 * 3 * nc * sv_elem(), ev);
        } else {
            FRetract<false> f;
            f.coef = d_coef_;
            pointwise(f, in, out);
        }
    }
    for (int i = 0; i < 3; ++i) {
        for (int j = -1; j < 3 && !from_retraction; ++j) {
            InvOut o;
            o.nsrc = 1;
            o.src[0] = ZSrc{scomp(u, i), sf64(), j < 0 ? SYM_ONE : SYM_IKX + j, 0, 1.0};
            o.phys_out = j < 0 ? PU + i : PD + 3 * i + j;
            io.push_back(o);
        }
        InvOut o;
        o.nsrc = 1;
        o.src[0] = ZSrc{scomp(u, i), sf64(), SYM_NEG_KSQ, 0, 1.0};  // laplacian (3248-3282)
        o.phys_out = PL + i;
        io.push_back(o);
    }
    inv(b, io);
    std::vector<int> uin;
    for (int i = 0; i < 3; ++i) uin.push_back(PU + i);
    for (int i = 0; i < 9; ++i) uin.push_back(PD + i);
    // 2. S -> P2, Q -> p spectrum (1102-1107)
    {
        FwdOut oS, oQ;
        oS.phys_out = PS;
        oS.spec = wspec(WS);
        oS.spec_f64 = wf64<T>();
        oQ.sym = SYM_INV_KSQ;
        oQ.spec = wspec(WP);
        oQ.spec_f64 = wf64<T>();
        if (from_retraction) {
            // Q of u = cs (u_prev + tau d) is cs^2 (Q_0 + tau Q_1 + tau^2 Q_2),
            // the line search's coefficient spectra (same symbol)
            const long nsp = (long)b.nb * b.nb * b.nx;
            cudaEvent_t ev = prof_mark();
            spec_poly3_kernel<cpx<T>><<<grid_for(nsp, 256), 256, 0, stream>>>(
                wspec(WP), wspec(WLQ), wspec(WLQ + 1), wspec(WLQ + 2), nsp, 0.0, 0.0, 0.0, d_coef_);
            launched("spec_poly", 4.0 * nsp * sizeof(cpx<T>), ev);
            if (!sac) fwd(b, FSq3{}, {PU, PU + 1, PU + 2}, {oS});
        } else {
            fwd(b, FG1{}, uin, {oS, oQ});
        }
    }
    // 3. grad p (1109)
    {
        std::vector<InvOut> g;
        for (int j = 0; j < 3; ++j) {
            InvOut o;
            o.nsrc = 1;
            o.src[0] = ZSrc{wspec(WP), wf64<T>(), SYM_IKX + j, 0, 1.0};
            o.phys_out = PGP + j;
            g.push_back(o);
        }
        inv(b, g);
    }
    // 4. |u|^k fields
    if (!sac) A_and_S(true);
    PowField a2 = chain(q - 2.0);
    PowField a4;
    if (!use_e_u) a4 = chain(q - 4.0);
    PowField ah = chain(q / 2.0);
    ensure_phys(a2);
    // 5. aux2 and c = P2(a2 u) (1115-1153)
    {
        FwdOut oT, oc[3];
        oT.phys_out = PT;
        for (int i = 0; i < 3; ++i) {
            oc[i].spec = scomp(c, i);
            oc[i].spec_f64 = sf64();
        }
        std::vector<int> in2;
        for (int i = 0; i < 3; ++i) in2.push_back(PU + i);
        for (int i = 0; i < 3; ++i) in2.push_back(PL + i);
        for (int i = 0; i < 3; ++i) in2.push_back(PGP + i);
        in2.push_back(a2.phys);
        if (sac) {
            FG2T f;
            f.cvisc = cv;
            f.cpress = cp;
            fwd(b, f, std::vector<int>(in2.begin(), in2.begin() + 9), {oT});
        } else if (!use_e_u) {
            FG2 f;
            f.cvisc = cv;
            f.cpress = cp;
            fwd(b, f, in2, {oT, oc[0], oc[1], oc[2]});
            if (a4.kind != PowField::ONE) {
                ensure_phys(a4);
                FwdOut o;
                o.phys_out = PT;
                fwd(b, FMul{}, {a4.phys, PT}, {o});
            }
        } else {
            FG2E f;
            f.cvisc = cv;
            f.cpress = cp;
            in2.push_back(PS);
            fwd(b, f, in2, {oT, oc[0], oc[1], oc[2]});
            FwdOut o;
            o.phys_out = PT;
            fwd(b, FMul{}, {a2.phys, PT}, {o});
        }
    }
    // 6. grad aux4 = grad Lap^-1 div c (1155-1158): the scalar spectrum
    // D = -i (K_odd . c) / |K|^2 once, then its three gradients i K_odd,k D
    // (= K_odd,k (K_odd . c) / |K|^2) from one load of D per column
    {
        const SpecGeom g2 = geom(b);
        cudaEvent_t ev = prof_mark();
        if (state32_)
            spec_div_ksq_kernel<float2, T><<<grid_for(g2.ncomp, 256), 256, 0, stream>>>(
                g2, (const float2*)scomp(c, 0), (const float2*)scomp(c, 1), (const float2*)scomp(c, 2), wspec(WDIV));
        else
            spec_div_ksq_kernel<double2, T><<<grid_for(g2.ncomp, 256), 256, 0, stream>>>(
                g2, (const double2*)scomp(c, 0), (const double2*)scomp(c, 1), (const double2*)scomp(c, 2),
                wspec(WDIV));
        launched("spec_scale", (double)g2.ncomp * (3.0 * sv_elem() + sizeof(cpx<T>)), ev);
        std::vector<InvOut> gi;
        for (int k = 0; k < 3; ++k) {
            InvOut o;
            o.nsrc = 1;
            o.src[0] = ZSrc{wspec(WDIV), wf64<T>(), SYM_IKX + k, 0, 1.0};
            o.phys_out = PGA + k;
            gi.push_back(o);
        }
        inv(b, gi);
    }
    // 7. final sum, one dealias, plus vc nu Lap c (1172-1190)
    {
        std::vector<int> in3;
        in3.push_back(PT);
        for (int i = 0; i < 3; ++i) in3.push_back(PU + i);
        in3.push_back(a2.phys);
        for (int i = 0; i < 3; ++i) in3.push_back(PGP + i);
        for (int i = 0; i < 9; ++i) in3.push_back(PD + i);
        for (int i = 0; i < 3; ++i) in3.push_back(PGA + i);
        for (int i = 0; i < 3; ++i) in3.push_back(PL + i);
        FwdOut o[3];
        for (int i = 0; i < 3; ++i) {
            o[i].spec = scomp(v, i);
            o[i].spec_f64 = sf64();
            o[i].add = scomp(c, i);
            o[i].add_f64 = sf64();
            o[i].add_sym = SYM_NEG_KSQ;
            o[i].add_coef = cv;
        }
        if (!use_e_u) {
            FG3<false> f;
            f.qm2 = q - 2.0;
            f.cvisc = cv;
            f.cpress = cp;
            fwd(b, f, in3, {o[0], o[1], o[2]});
        } else {
            FG3<true> f;
            f.qm2 = q - 2.0;
            f.cvisc = cv;
            f.cpress = cp;
            in3.push_back(PS);
            fwd(b, f, in3, {o[0], o[1], o[2]});
        }
    }
    if (want_lq) {
        if (ah.kind == PowField::RAW || ah.spec < 0) {
            pointwise(FSqRed{}, {ah.phys}, {}, 20);
            grad_lq_slot_ = 20;
        } else {
            ensure_p2_spec(ah);
            sdots(*this, {{wspec(ah.spec), wspec(ah.spec)}}, 0);
            grad_lq_slot_ = 0;
        }
    }
}

// ||u + tau d||_q^q (calc_global_Lq_norm)
template <typename T>
double Engine<T>::lq_pow(const SVec* u, const SVec* d, double tau) {
    pu_of_ = nullptr;
    const long nc = spec_ncomp();
    chain_reset();
    if (!w_from_memo(u, d, tau)) {
        std::vector<InvOut> io;
        for (int i = 0; i < 3; ++i) {
            InvOut o;
            o.nsrc = d ? 2 : 1;
            o.src[0] = ZSrc{scomp(u, i), sf64(), SYM_ONE, 0, 1.0};
            if (d) o.src[1] = ZSrc{scomp(d, i), sf64(), SYM_ONE, 0, tau};
            o.phys_out = PU + i;
            io.push_back(o);
        }
        inv(b2, io);
    }
    FwdOut oS;
    oS.phys_out = PS;
    fwd(b2, FSq3{}, {PU, PU + 1, PU + 2}, {oS});
    A_and_S(true);
    PowField ah = chain(P.q / 2.0);
    if (ah.kind == PowField::RAW || ah.spec < 0) {
        pointwise(FSqRed{}, {ah.phys}, {}, 20);
        fetch_results();
        return h_results[20];
    }
    ensure_p2_spec(ah);
    sdots(*this, {{wspec(ah.spec), wspec(ah.spec)}}, 0);
    fetch_results();
    return h_results[0];
}

// vectorTransport (function_ops.f90:1716-1768) pieces at w = u + tau d.
template <typename T>
double Engine<T>::transport_pieces(const SVec* u, const SVec* d, double tau, const SVec* const* xi,
                                   int nxi, double* ir) {
    pu_of_ = nullptr;
    const long nc = spec_ncomp();
    const double q = P.q;
    chain_reset();
    const bool memo = w_from_memo(u, d, tau);
    if (!memo) {
        std::vector<InvOut> io;
        for (int i = 0; i < 3; ++i) {
            InvOut o;
            o.nsrc = d ? 2 : 1;
            o.src[0] = ZSrc{scomp(u, i), sf64(), SYM_ONE, 0, 1.0};
            if (d) o.src[1] = ZSrc{scomp(d, i), sf64(), SYM_ONE, 0, tau};
            o.phys_out = PU + i;
            io.push_back(o);
        }
        inv(b2, io);
    }
    const PhysMemo m = pm_;  // this program's own writes below keep it
    if (memo && q == 4.0 && !use_e_u && ls_clamp_free(tau)) {
        // |w|^2 = S_0 + tau S_1 + tau^2 S_2 (the line search's coefficient
        // fields, P2 linear) is >= 0 at every point, so A = P2(max(S, 0)) = S
        FPolyS f;
        f.tau = tau;
        pointwise(f, {ls_phys(0), ls_phys(1), ls_phys(2)}, {PS, PA});
        const long nsp = (long)b2.nb * b2.nb * b2.nx;
        cudaEvent_t ev = prof_mark();
        spec_poly3_kernel<cpx<T>><<<grid_for(nsp, 256), 256, 0, stream>>>(
            wspec(WS), wspec(ls_wspec(0)), wspec(ls_wspec(1)), wspec(ls_wspec(2)), nsp, 1.0, tau, tau * tau, nullptr);
        launched("spec_poly", 4.0 * nsp * sizeof(cpx<T>), ev);
        MLQ_CUDA(cudaMemcpyAsync(wspec(WA), wspec(WS), nsp * sizeof(cpx<T>), cudaMemcpyDeviceToDevice, stream));
    } else {
        FwdOut oS;
        oS.phys_out = PS;
        oS.spec = wspec(WS);
        oS.spec_f64 = wf64<T>();
        fwd(b2, FSq3{}, {PU, PU + 1, PU + 2}, {oS});
        A_and_S(true);
    }
    PowField a2 = chain(q - 2.0);
    PowField ah = chain(q / 2.0);
    if (!c_tmp_) c_tmp_ = alloc_state();
    SVec* cbuf = c_tmp_;
    if (q - 2.0 > MACH_EPSILON) {
        // aux = P2(|w|^{q-2} w) (1737-1740)
        ensure_phys(a2);
        FwdOut o[3];
        for (int i = 0; i < 3; ++i) {
            o[i].spec = scomp(cbuf, i);
            o[i].spec_f64 = sf64();
        }
        fwd(b2, FC3{}, {a2.phys, PU, PU + 1, PU + 2}, {o[0], o[1], o[2]});
        if (memo) {
            pm_ = m;
            // at q = 4 (no e_u) the gradient's S, A = |u|^{q-2} and c are these
            pm_.sac = q == 4.0 && !use_e_u && a2.phys == PA && a2.spec == WA;
        }
    } else {
        if (a2.kind != PowField::ONE) throw CudaError("vectorTransport with 2 < q < 2+eps", MLQ_ERR_BADARG);
        lincomb(cbuf, 1.0, u, d ? tau : 0.0, d, 0.0, nullptr);
    }
    double lqq;
    if (ah.kind == PowField::RAW || ah.spec < 0) {
        pointwise(FSqRed{}, {ah.phys}, {}, 20);
        fetch_results();
        lqq = h_results[20];
    } else {
        ensure_p2_spec(ah);
        sdots(*this, {{wspec(ah.spec), wspec(ah.spec)}}, 0);
        fetch_results();
        lqq = h_results[0];
    }
    for (int k = 0; k < nxi; k += 6) {
        SpecDotPair pr[6];
        const int m = std::min(6, nxi - k);
        for (int i = 0; i < m; ++i) pr[i] = SpecDotPair{cbuf, xi[k + i], 0};
        dots(pr, m, ir + k);
    }
    return lqq;
}

// calc_uk (function_ops.f90:2324-2343) of the state u into phys(dst)
template <typename T>
void Engine<T>::calc_uk(const SVec* u, double k, int dst) {
    pu_of_ = nullptr;
    const long nc = spec_ncomp();
    chain_reset();
    std::vector<InvOut> io;
    for (int i = 0; i < 3; ++i) {
        InvOut o;
        o.nsrc = 1;
        o.src[0] = ZSrc{scomp(u, i), sf64(), SYM_ONE, 0, 1.0};
        o.phys_out = PU + i;
        io.push_back(o);
    }
    inv(b2, io);
    FwdOut oS;
    oS.phys_out = PS;
    fwd(b2, FSq3{}, {PU, PU + 1, PU + 2}, {oS});
    A_and_S(true);
    PowField f = chain(k);
    ensure_phys(f);
    if (slab_) {
        const PSlot src = slot(f.phys);
        slot(dst) = src;
        if (src.kind == PSlot::YS)
            MLQ_CUDA(cudaMemcpyAsync(slot_ys(dst), slot_ys_[f.phys], (size_t)n * src.band.nb * px_of(src.band) * sizeof(cpx<T>),
                                     cudaMemcpyDeviceToDevice, stream));
        return;
    }
    MLQ_CUDA(cudaMemcpyAsync(phys(dst), phys(f.phys), n3 * sizeof(T), cudaMemcpyDeviceToDevice, stream));
}

// ----------------------------------------------------------------------------
// line search along phi = u + tau d at q = 4
// ----------------------------------------------------------------------------

// Per block: the largest lower end and the smallest upper end, over its
// points, of the interval around tau = 0 on which s0 + tau s1 + tau^2 s2 >= 0
// (empty when s0 < 0), then the same around each anchor (empty where S is
// negative at the anchor), as (lo, hi) pairs: 2 (LS_ANCHORS + 1) per block.
template <typename T>
__global__ void __launch_bounds__(RED_THREADS, 4)
    ls_interval_kernel(const T* __restrict__ s0, const T* __restrict__ s1, const T* __restrict__ s2, long npts,
                       LsAnchorSet an, double* __restrict__ out) {
    constexpr int K = LS_ANCHORS + 1;
    const double inf = 1e300;
    double lo[K], hi[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        lo[k] = -inf;
        hi[k] = inf;
    }
    auto point = [&](double a, double b, double c) {
        // S > 0 for every tau (upward, no real root) or constant >= 0: no
        // point constraint, nothing to reduce (most points)
        if ((a > 0.0 && b * b - 4.0 * a * c < 0.0) || (a == 0.0 && b == 0.0 && c >= 0.0)) return;
        const LsRoots r = ls_roots(a, b, c);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double l, h;
            if (k == 0)
                ls_component0(r, a, b, c, l, h);
            else
                ls_component(r, a, b, c, an.a[k - 1], l, h);
            lo[k] = fmax(lo[k], l);
            hi[k] = fmin(hi[k], h);
        }
    };
    // two points per pass: both points' loads are in flight together
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += 2 * stride) {
        const bool two = i + stride < npts;
        const long j = two ? i + stride : i;
        const double a0 = (double)s2[i], b0 = (double)s1[i], c0 = (double)s0[i];
        const double a1 = (double)s2[j], b1 = (double)s1[j], c1 = (double)s0[j];
        point(a0, b0, c0);
        if (two) point(a1, b1, c1);
    }
    __shared__ double slo[K][RED_THREADS / 32], shi[K][RED_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fmax(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
            hi[k] = fmin(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
        }
        if (lane == 0) {
            slo[k][warp] = lo[k];
            shi[k][warp] = hi[k];
        }
    }
    __syncthreads();
    if (threadIdx.x < K) {
        const int k = threadIdx.x;
        double l = slo[k][0], h = shi[k][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            l = fmax(l, slo[k][w]);
            h = fmin(h, shi[k][w]);
        }
        out[2 * K * blockIdx.x + 2 * k] = l;
        out[2 * K * blockIdx.x + 2 * k + 1] = h;
    }
}

// Per block: the minimum over its points of s0 + tau (s1 + tau s2), evaluated
// exactly as the trial functor FLSA does (precision T).
template <typename T>
__global__ void __launch_bounds__(RED_THREADS)
    ls_min_kernel(const T* __restrict__ s0, const T* __restrict__ s1, const T* __restrict__ s2, long npts, double tau,
                  const double* __restrict__ taup, double* __restrict__ out) {
    const T t = (T)(taup ? *taup : tau);
    T m = T(1e30);
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += (long)gridDim.x * blockDim.x)
        m = fmin(m, s0[i] + t * (s1[i] + t * s2[i]));
    __shared__ T sm[RED_THREADS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmin(m, sm[w]);
        out[blockIdx.x] = (double)m;
    }
}

template <typename T>
void Engine<T>::ls_setup(const SVec* u, const SVec* d, double tau0) {
    const long nc = spec_ncomp();
    ls_free_val_ = -1;
    ls_dev_ = ls_device_ready();
    if (ls_dev_ && !d_ls_) {
        d_ls_ = (LsDevState*)dev_alloc(sizeof(LsDevState));
        MLQ_CUDA(cudaMallocHost(&h_ls_, 1024));
    }
    // u and grad u are still in PU, PD when the gradient program of this
    // iteration transformed the same spectrum
    const bool reuse_u = !slab_ && reuse_on_ && pu_of_ == (const void*)u;
    if (slab_) release_slots(0, LU);  // the programs' fields are rebuilt by the next program
    const int iu = reuse_u ? (int)PU : (int)LU, idu = reuse_u ? (int)PD : (int)LDU;
    // phi's pieces: u, d and their gradients (function_ops.f90:3147-3195)
    std::vector<InvOut> io;
    for (int f = reuse_u ? 1 : 0; f < 2; ++f)
        for (int i = 0; i < 3; ++i)
            for (int j = -1; j < 3; ++j) {
                InvOut o;
                o.nsrc = 1;
                o.src[0] = ZSrc{scomp(f == 0 ? u : d, i), sf64(), j < 0 ? SYM_ONE : SYM_IKX + j, 0, 1.0};
                o.phys_out = j < 0 ? (f == 0 ? LU : LD) + i : (f == 0 ? LDU : LDD) + 3 * i + j;
                io.push_back(o);
            }
    inv(b2, io);
    if (!slab_ && reuse_on_) {
        pm_ = PhysMemo{};
        pm_.u = u;
        pm_.d = d;
        pm_.iu = iu;
        pm_.idu = idu;
        pm_.ls = true;
    }
    std::vector<int> ud = {iu, iu + 1, iu + 2, LD, LD + 1, LD + 2};
    std::vector<int> all;
    for (int i = 0; i < 3; ++i) all.push_back(iu + i);
    for (int i = 0; i < 9; ++i) all.push_back(idu + i);
    for (int i = 0; i < 3; ++i) all.push_back(LD + i);
    for (int i = 0; i < 9; ++i) all.push_back(LDD + i);
    std::vector<int> grads;
    for (int i = 0; i < 9; ++i) grads.push_back(idu + i);
    for (int i = 0; i < 9; ++i) grads.push_back(LDD + i);
    // P2 of the coefficients of |phi|^2 (calc_uk 2332-2333).  The tau^0 one,
    // P2(|u|^2), is the gradient program's S when it ran for this u.
    {
        const bool s0 = !slab_ && reuse_on_ && ws_of_ == (const void*)u;
        ls_p0_ = s0 ? (int)PS : (int)LS;
        ls_w0_ = s0 ? WS : WLS;
        FwdOut o[3];
        for (int a = 0; a < 3; ++a) {
            o[a].phys_out = LS + a;
            o[a].spec = wspec(WLS + a);
            o[a].spec_f64 = wf64<T>();
        }
        if (s0)
            fwd(b2, FLSS12{}, ud, {o[1], o[2]});
        else
            fwd(b2, FLSS{}, ud, {o[0], o[1], o[2]});
    }
    // P2 of the coefficients of W_j = sum_i phi_i d_j phi_i (calc_vgraduvgradu /
    // calc_vvgradu, v = phi).  W_j = (1/2) d_j |phi|^2, and when the cut c
    // satisfies 3c < N the dealiased grid product of two band-limited fields
    // is the band truncation of their exact product (its aliases land beyond
    // the cut), so P2(W_j) = (1/2) d_j P2(|phi|^2): the derivatives of the
    // S_a spectra just formed.  For 3c >= N (N divisible by 3) the products
    // are formed and dealiased as the reference does.
    if (reuse_on_ && 3 * b2.cut < n) {
        std::vector<InvOut> g;
        for (int a = 0; a < 3; ++a)
            for (int j = 0; j < 3; ++j) {
                InvOut o;
                o.nsrc = 1;
                o.src[0] = ZSrc{wspec(ls_wspec(a)), wf64<T>(), SYM_IKX + j, 0, 0.5};
                o.phys_out = LV + 3 * a + j;
                g.push_back(o);
            }
        inv(b2, g);
    } else {
        std::vector<int> uself(all.begin(), all.begin() + 12), dself(all.begin() + 12, all.end());
        FwdOut o[3];
        for (int j = 0; j < 3; ++j) o[j].phys_out = LV + j;
        fwd(b2, FLSW<0>{}, uself, {o[0], o[1], o[2]});
        for (int j = 0; j < 3; ++j) o[j].phys_out = LV + 3 + j;
        fwd(b2, FLSW<1>{}, all, {o[0], o[1], o[2]});
        for (int j = 0; j < 3; ++j) o[j].phys_out = LV + 6 + j;
        fwd(b2, FLSW<0>{}, dself, {o[0], o[1], o[2]});
    }
    // p_a = -Lap^-1 P2(Q_a) and the spectra of P2(|grad phi|^2)_a
    {
        FwdOut o[6];
        for (int a = 0; a < 3; ++a) {
            o[a].sym = SYM_INV_KSQ;
            o[a].phys_out = LP + a;
            if (!slab_) {  // the next gradient's pressure source is a polynomial in tau of these
                o[a].spec = wspec(WLQ + a);
                o[a].spec_f64 = wf64<T>();
            }
            o[3 + a].spec = wspec(WLG + a);
            o[3 + a].spec_f64 = wf64<T>();
        }
        fwd(b2, FLSQG{}, grads, {o[0], o[1], o[2], o[3], o[4], o[5]});
    }
    // R2 and R3 integrands as polynomials in tau
    std::vector<int> rin;
    for (int i = 0; i < 9; ++i) rin.push_back(LV + i);
    for (int a = 0; a < 3; ++a) rin.push_back(LP + a);
    for (int i = 0; i < 6; ++i) rin.push_back(ud[i]);
    pointwise(FLSRed{}, rin, {}, 100);
    if (!ls_dev_) fetch_results();
    if (slab_) {  // the trials read only S_a
        release_slots(LU, LS);
        release_slots(LV, LP + 3);
    }
    // Parseval products for the transform-free trials
    {
        std::vector<std::pair<const cpx<T>*, const cpx<T>*>> p1, p2, p3;
        for (int i = 0; i < 3; ++i)
            for (int a = 0; a < 3; ++a) (i < 2 ? p1 : p2).push_back({wspec(ls_wspec(i)), wspec(WLG + a)});
        for (int i = 0; i < 3; ++i)
            for (int j = i; j < 3; ++j)
                (p2.size() < 6 ? p2 : p3).push_back({wspec(ls_wspec(i)), wspec(ls_wspec(j))});
        sdots(*this, p1, 140);
        sdots(*this, p2, 146);
        sdots(*this, p3, 152);
    }
    // the interval of tau around 0 on which S(tau) >= 0 everywhere
    LsAnchorSet an;
    ls_anchors(tau0, an.a);
    constexpr int W = 2 * (LS_ANCHORS + 1);  // interval ends per block
    if (ls_dev_) {
        // on the device, with the coefficients: no host round trip
        const int grid = grid_for(n3, RED_THREADS, 148 * 4);
        ensure_partials((long)grid * W);
        cudaEvent_t ev = prof_mark();
        ls_interval_kernel<T><<<grid, RED_THREADS, 0, stream>>>(phys(ls_phys(0)), phys(ls_phys(1)),
                                                                phys(ls_phys(2)), n3, an, d_partials);
        launched("ls_interval", 3.0 * n3 * sizeof(T), ev);
        ls_launch_coef(d_ls_, d_results, d_partials, grid, an, stream);
        launched();
        ls_host_poly_ = false;
        return;
    }
    double lo[LS_ANCHORS + 1], hi[LS_ANCHORS + 1];
    for (int k = 0; k <= LS_ANCHORS; ++k) {
        lo[k] = -1e300;
        hi[k] = 1e300;
    }
    {
        const long npts = slab_ ? (long)zs_ * n * n : n3;
        const int grid = grid_for(npts, RED_THREADS, 148 * 4);
        ensure_partials((long)grid * W);
        std::vector<double> h((size_t)grid * W);
        for (int z0 = 0; z0 < n; z0 += (slab_ ? zs_ : n)) {
            const T* s[3];
            if (slab_) {
                const std::vector<const T*> p = expand_many({ls_phys(0), ls_phys(1), ls_phys(2)}, z0);
                for (int a = 0; a < 3; ++a) s[a] = p[a];
            } else {
                for (int a = 0; a < 3; ++a) s[a] = phys(ls_phys(a));
            }
            ls_interval_kernel<T><<<grid, RED_THREADS, 0, stream>>>(s[0], s[1], s[2], npts, an, d_partials);
            launched();
            MLQ_CUDA(cudaMemcpyAsync(h.data(), d_partials, h.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
            MLQ_CUDA(cudaStreamSynchronize(stream));
            for (int g = 0; g < grid; ++g)
                for (int k = 0; k <= LS_ANCHORS; ++k) {
                    lo[k] = fmax(lo[k], h[W * g + 2 * k]);
                    hi[k] = fmin(hi[k], h[W * g + 2 * k + 1]);
                }
        }
    }
    fetch_results();
    // <S_i, G_a> in slots 140..148 (146.. holds i = 2), <S_i, S_j> in 149..154
    ls_assemble(h_results + 100, h_results + 140, h_results + 149, lo[0], hi[0], lo + 1, hi + 1, an.a, ls_c_);
    ls_host_poly_ = true;
}

template <typename T>
void Engine<T>::ls_poly_to_host() {
    if (ls_host_poly_) return;
    LsPoly* hp = (LsPoly*)((char*)h_ls_ + 512);
    MLQ_CUDA(cudaMemcpyAsync(hp, &d_ls_->poly, sizeof(LsPoly), cudaMemcpyDeviceToHost, stream));
    MLQ_CUDA(cudaStreamSynchronize(stream));
    ls_c_ = *hp;
    ls_host_poly_ = true;
}

// the only node of a captured sequence without successors
static cudaGraphNode_t graph_leaf(cudaGraph_t g) {
    size_t nn = 0;
    MLQ_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    MLQ_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
    cudaGraphNode_t leaf = nullptr;
    int nleaf = 0;
    for (cudaGraphNode_t x : nodes) {
        size_t nd = 0;
        MLQ_CUDA(cudaGraphNodeGetDependentNodes(x, nullptr, &nd));
        if (nd == 0) {
            leaf = x;
            ++nleaf;
        }
    }
    if (nleaf != 1) throw CudaError("line-search graph: captured sequence is not a chain", MLQ_ERR_CUDA);
    return leaf;
}

// an If (or While) node after dep (or at the root) of g; returns its body
static cudaGraph_t add_conditional(cudaGraph_t g, cudaGraphNode_t dep, cudaGraphConditionalHandle h,
                                   cudaGraphConditionalNodeType type) {
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = type;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    MLQ_CUDA(cudaGraphAddNode(&node, g, dep ? &dep : nullptr, dep ? 1 : 0, &np));
    return np.conditional.phGraph_out[0];
}

// The device search as one graph:
//   while (h_loop) { ctrl; if (h_chk) { ls_min; check; if (h_fft) { transform trial; fft } } }
// Each conditional handle is set by a kernel of the graph that holds its node
// (the loop's by the controller in its body).  The controller ends the loop
// after LS_MAX_LOOPS passes, so the loop is bounded whatever the kernels see.
template <typename T>
bool Engine<T>::ls_graph_build(LsGraph& g, int key) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    const int grid = grid_for(n3, RED_THREADS, 148 * 4);
    ensure_partials((long)grid * 2);
    FwdOut o;
    o.red_self = 0;
    for (int a = 0; a < 3; ++a) {
        o.red_with[a] = wspec(WLG + a);
        o.red_with_f64[a] = wf64<T>();
        o.red_with_slot[a] = 1 + a;
    }
    const std::vector<int> in = {ls_phys(0), ls_phys(1), ls_phys(2)};
    const bool prof_was = prof_on;
    prof_on = false;
    // one transform trial run directly, so that the buffers it allocates on
    // first use exist before the capture (its sums land in unused slots)
    FLSA f0;
    f0.tau = 0.0;
    const long long l0 = launches;
    bool ok = true;
    try {
        fwd(b2, f0, in, {o}, 130);
    } catch (...) {
        ok = false;
    }
    const long long nfwd = launches - l0;
    cudaGraph_t G = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto capture_into = [&](cudaGraph_t body, auto&& fn) {
        MLQ_CUDA(cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        bool fine = true;
        try {
            fn();
        } catch (...) {
            fine = false;
        }
        cudaGraph_t got = nullptr;
        const cudaError_t e = cudaStreamEndCapture(stream, &got);
        if (!fine || e != cudaSuccess || got != body)
            throw CudaError("line-search graph: capture failed", MLQ_ERR_CUDA);
    };
    if (ok) try {
            MLQ_CUDA(cudaGraphCreate(&G, 0));
            cudaGraphConditionalHandle h_loop, h_chk, h_fft;
            MLQ_CUDA(cudaGraphConditionalHandleCreate(&h_loop, G, 1, cudaGraphCondAssignDefault));
            cudaGraph_t body_loop = add_conditional(G, nullptr, h_loop, cudaGraphCondTypeWhile);
            MLQ_CUDA(cudaGraphConditionalHandleCreate(&h_chk, body_loop, 0, cudaGraphCondAssignDefault));
            capture_into(body_loop, [&] { ls_launch_ctrl(d_ls_, h_loop, h_chk, stream); });
            cudaGraph_t body_chk = add_conditional(body_loop, graph_leaf(body_loop), h_chk, cudaGraphCondTypeIf);
            MLQ_CUDA(cudaGraphConditionalHandleCreate(&h_fft, body_chk, 0, cudaGraphCondAssignDefault));
            capture_into(body_chk, [&] {
                ls_min_kernel<T><<<grid, RED_THREADS, 0, stream>>>(phys(in[0]), phys(in[1]), phys(in[2]), n3, 0.0,
                                                                   &d_ls_->ptau, d_partials);
                ls_launch_check(d_ls_, d_partials, grid, h_fft, stream);
            });
            cudaGraph_t body_fft = add_conditional(body_chk, graph_leaf(body_chk), h_fft, cudaGraphCondTypeIf);
            capture_into(body_fft, [&] {
                FLSA f;
                f.tau = 0.0;
                f.taup = &d_ls_->ptau;
                fwd(b2, f, in, {o}, 130);
                ls_launch_fft(d_ls_, d_results + 130, stream);
            });
            MLQ_CUDA(cudaGraphInstantiate(&exec, G, 0));
        } catch (...) {
            ok = false;
        }
    if (G) cudaGraphDestroy(G);
    cudaGetLastError();
    launches = l0 + nfwd;  // captured launches did not run
    prof_on = prof_was;
    if (!ok) {
        if (exec) cudaGraphExecDestroy(exec);
        return false;
    }
    g.exec = exec;
    g.gen = graph_gen_;
    g.key = key;
    g.nfwd = nfwd;
    return true;
}

template <typename T>
int Engine<T>::ls_device_search(double B, double tA0, double tB0, LsOut* out) {
    if (!ls_dev_) return 1;
    const int key = ls_phys(0);
    LsGraph* g = nullptr;
    for (LsGraph& x : lsg_)
        if (x.exec && x.key == key && x.gen == graph_gen_) g = &x;
    if (!g) {
        g = &lsg_[0];
        for (LsGraph& x : lsg_)
            if (!x.exec || x.gen != graph_gen_) {
                g = &x;
                break;
            }
        if (!ls_graph_build(*g, key)) {
            lsg_failed_ = true;
            return 1;
        }
    }
    char* h = (char*)h_ls_;
    LsParams* hp = (LsParams*)h;
    *hp = LsParams{P.q, P.visc_coef * P.visc, P.press_coef, B, tA0, tB0, ls_transform_trials_ ? 1 : 0};
    MLQ_CUDA(cudaMemcpyAsync(&d_ls_->par, hp, sizeof(LsParams), cudaMemcpyHostToDevice, stream));
    cudaEvent_t ev = prof_mark();
    MLQ_CUDA(cudaGraphLaunch(g->exec, stream));
    launched("line_search", 0.0, ev);
    LsOut* ho = (LsOut*)(h + 256);
    LsPoly* hpoly = (LsPoly*)(h + 512);
    MLQ_CUDA(cudaMemcpyAsync(ho, &d_ls_->out, sizeof(LsOut), cudaMemcpyDeviceToHost, stream));
    MLQ_CUDA(cudaMemcpyAsync(hpoly, &d_ls_->poly, sizeof(LsPoly), cudaMemcpyDeviceToHost, stream));
    fetch_results();  // the transform trials' NaN flag
    ls_c_ = *hpoly;
    ls_host_poly_ = true;
    *out = *ho;
    // the graph's kernels (one launch counted above)
    launches += out->loops + 2LL * out->checks + out->nfft * (g->nfwd + 1) - 1;
    ++ls_dev_searches_;
    ls_dev_loops_ += out->loops;
    ls_poly_trials_ += out->npoly;
    ls_fft_trials_ += out->nfft;
    if (out->status == 0 && out->mflag == 0) {
        ls_free_tau_ = out->tau1;
        ls_free_val_ = out->fft1 ? 0 : 1;
    }
    return 0;
}

template <typename T>
bool Engine<T>::ls_clamp_free(double tau) {
    if (ls_free_val_ >= 0 && tau == ls_free_tau_) return ls_free_val_ != 0;  // decided by the device search
    if (ls_transform_trials_) return false;
    ls_poly_to_host();
    bool clamp_off = ls_free(ls_c_, tau);
    if (!clamp_off) {
        // outside the interval: one read of S_0..2 decides for this tau
        const long npts = slab_ ? (long)zs_ * n * n : n3;
        const int grid = grid_for(npts, RED_THREADS, 148 * 4);
        ensure_partials(grid);
        std::vector<double> h(grid);
        double mn = 1e300;
        for (int z0 = 0; z0 < n; z0 += (slab_ ? zs_ : n)) {
            const T* sp[3];
            if (slab_) {
                const std::vector<const T*> p = expand_many({ls_phys(0), ls_phys(1), ls_phys(2)}, z0);
                for (int a = 0; a < 3; ++a) sp[a] = p[a];
            } else {
                for (int a = 0; a < 3; ++a) sp[a] = phys(ls_phys(a));
            }
            cudaEvent_t ev = prof_mark();
            ls_min_kernel<T><<<grid, RED_THREADS, 0, stream>>>(sp[0], sp[1], sp[2], npts, tau, nullptr, d_partials);
            launched("ls_min", 3.0 * npts * sizeof(T), ev);
            MLQ_CUDA(cudaMemcpyAsync(h.data(), d_partials, h.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
            MLQ_CUDA(cudaStreamSynchronize(stream));
            for (double v : h) mn = std::min(mn, v);
        }
        clamp_off = mn >= 0.0;
    }
    return clamp_off;
}

template <typename T>
void Engine<T>::ls_trial(double tau, double out[3], double* lqq) {
    const double q = P.q, cv = P.visc_coef * P.visc, cp = P.press_coef;
    double l = 0.0;
    if (ls_clamp_free(tau)) {
        // S(tau) >= 0 everywhere: P2(g^2) = S(tau), every product is a polynomial
        ++ls_poly_trials_;
        ls_poly_R(ls_c_, q, cv, cp, tau, out, &l);
        if (lqq) *lqq = l;
        return;
    }
    ++ls_fft_trials_;
    // A(tau) = P2(g^2) with its Parseval products: ||A||^2 (= ||phi||_4^4) and
    // <A, P2(|grad phi|^2)_a>, a = 0..2
    FwdOut o;
    o.red_self = 0;
    for (int a = 0; a < 3; ++a) {
        o.red_with[a] = wspec(WLG + a);
        o.red_with_f64[a] = wf64<T>();
        o.red_with_slot[a] = 1 + a;
    }
    FLSA f;
    f.tau = tau;
    fwd(b2, f, {ls_phys(0), ls_phys(1), ls_phys(2)}, {o}, 130);
    fetch_results();
    ls_fft_R(ls_c_, q, cv, cp, h_results + 130, tau, out, &l);
    if (lqq) *lqq = l;
}

// ----------------------------------------------------------------------------
// state <-> host
// ----------------------------------------------------------------------------
// Host copies of transfers run on several threads, and are pipelined with
// the DMA in chunks through two pinned staging buffers.
template <class Fn>
static void par_range(long count, Fn&& fn) {
    const long nt = std::max(1L, std::min<long>(16, (long)std::thread::hardware_concurrency() / 2));
    if (nt == 1 || count < (1L << 20)) {
        fn(0L, count);
        return;
    }
    std::vector<std::thread> th;
    const long per = (count + nt - 1) / nt;
    for (long t = 0; t < nt; ++t) {
        const long a = t * per, b = std::min(count, a + per);
        if (a < b) th.emplace_back([&fn, a, b] { fn(a, b); });
    }
    for (auto& x : th) x.join();
}

static constexpr long XFER_CHUNK = 1L << 25;  // elements per pipelined chunk

// A host buffer the caller allocated pinned (page-locked): the DMA engine
// reads and writes it directly, with no staging copy.
static bool host_pinned(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

template <typename T>
void Engine<T>::load_scalar_phys(const double* host, int dst, cudaStream_t xs) {
    const cudaStream_t st = (xs && !slab_) ? xs : stream;  // slab storage is filled on the engine's stream
    if (sizeof(T) == 8 && host_pinned(host)) {
        MLQ_CUDA(cudaMemcpyAsync(phys(dst), host, n3 * sizeof(T), cudaMemcpyHostToDevice, st));
        MLQ_CUDA(cudaStreamSynchronize(st));
        if (slab_) slot(dst).kind = PSlot::FULL;
        return;
    }
    const long ch = std::min(n3, XFER_CHUNK);
    T* buf[2];
    buf[0] = (T*)stage(2 * ch * sizeof(T));
    buf[1] = buf[0] + ch;
    cudaEvent_t done[2] = {ev_take(), ev_take()};
    T* d = phys(dst);
    long k = 0;
    for (long off = 0; off < n3; off += ch, ++k) {
        const long cnt = std::min(ch, n3 - off);
        T* b = buf[k & 1];
        if (k >= 2) MLQ_CUDA(cudaEventSynchronize(done[k & 1]));  // that buffer's DMA has finished
        par_range(cnt, [&](long a, long e) {
            if (sizeof(T) == 8)
                std::memcpy(b + a, host + off + a, (e - a) * sizeof(double));
            else
                for (long i = a; i < e; ++i) b[i] = (T)host[off + i];
        });
        MLQ_CUDA(cudaMemcpyAsync(d + off, b, cnt * sizeof(T), cudaMemcpyHostToDevice, st));
        MLQ_CUDA(cudaEventRecord(done[k & 1], st));
    }
    MLQ_CUDA(cudaStreamSynchronize(st));
    ev_give(done[0]);
    ev_give(done[1]);
    if (slab_) slot(dst).kind = PSlot::FULL;
}

template <typename T>
void Engine<T>::store_scalar_phys(int src, double* host, cudaStream_t xs) {
    const cudaStream_t st = (xs && !slab_) ? xs : stream;  // slab expansion runs on the engine's stream
    // chunks of whole slabs in slab mode (each expanded just before its copy)
    const long ch = slab_ ? (long)zs_ * n * n : std::min(n3, XFER_CHUNK);
    if (sizeof(T) == 8 && host_pinned(host)) {
        for (long off = 0; off < n3; off += ch) {
            const long cnt = std::min(ch, n3 - off);
            const T* d = slab_ ? expand(src, (int)(off / ((long)n * n)), 0) : phys(src) + off;
            MLQ_CUDA(cudaMemcpyAsync(host + off, d, cnt * sizeof(T), cudaMemcpyDeviceToHost, st));
        }
        MLQ_CUDA(cudaStreamSynchronize(st));
        return;
    }
    T* buf[2];
    buf[0] = (T*)stage(2 * ch * sizeof(T));
    buf[1] = buf[0] + ch;
    cudaEvent_t done[2] = {ev_take(), ev_take()};
    auto issue = [&](long k) {
        const long off = k * ch, cnt = std::min(ch, n3 - off);
        const T* d = slab_ ? expand(src, (int)(off / ((long)n * n)), 0) : phys(src) + off;
        MLQ_CUDA(cudaMemcpyAsync(buf[k & 1], d, cnt * sizeof(T), cudaMemcpyDeviceToHost, st));
        MLQ_CUDA(cudaEventRecord(done[k & 1], st));
    };
    const long nk = (n3 + ch - 1) / ch;
    for (long k = 0; k < std::min(nk, 2L); ++k) issue(k);
    for (long k = 0; k < nk; ++k) {
        const long off = k * ch, cnt = std::min(ch, n3 - off);
        MLQ_CUDA(cudaEventSynchronize(done[k & 1]));
        const T* b = buf[k & 1];
        par_range(cnt, [&](long a, long e) {
            if (sizeof(T) == 8)
                std::memcpy(host + off + a, b + a, (e - a) * sizeof(double));
            else
                for (long i = a; i < e; ++i) host[off + i] = (double)b[i];
        });
        if (k + 2 < nk) issue(k + 2);
    }
    MLQ_CUDA(cudaStreamSynchronize(st));
    ev_give(done[0]);
    ev_give(done[1]);
}

// Forward transform of a host vector field into band-b2 state spectra.  The
// energy the band drops is measured directly, as ||u - F^-1 P2 F u||^2.
// The second stream of host transfers (copies only), created on first use.
template <typename T>
cudaStream_t Engine<T>::copy_stream() {
    if (!xstream_) MLQ_CUDA(cudaStreamCreateWithFlags(&xstream_, cudaStreamNonBlocking));
    return xstream_;
}

// A host vector field in, component by component: each component is copied
// in on the copy stream while the engine's stream transforms the one before
// (two physical buffers in turn), then the band check's round trip.
template <typename T>
double Engine<T>::load_vec(const double* host, SVec* spec, int spec_f64) {
    const long nc = spec_ncomp();
    if (spec_f64 < 0) spec_f64 = sf64();
    const int bufs[2] = {PIO, PIO3};
    cudaStream_t xs = slab_ ? nullptr : copy_stream();
    cudaEvent_t used[2] = {ev_take(), ev_take()}, loaded = ev_take();
    // the buffers may still be read by work already on the engine's stream
    MLQ_CUDA(cudaEventRecord(used[0], stream));
    MLQ_CUDA(cudaEventRecord(used[1], stream));
    for (int c = 0; c < 3; ++c) {
        const int b = slab_ ? PIO : bufs[c & 1];
        if (xs) MLQ_CUDA(cudaStreamWaitEvent(xs, used[c & 1], 0));
        load_scalar_phys(host + c * n3, b, xs);
        if (xs) {
            MLQ_CUDA(cudaEventRecord(loaded, xs));
            MLQ_CUDA(cudaStreamWaitEvent(stream, loaded, 0));
        }
        FwdOut o;
        o.spec = (char*)spec + (size_t)c * nc * (spec_f64 ? sizeof(double2) : sizeof(float2));
        o.spec_f64 = spec_f64;
        o.phys_out = PIO2;
        fwd(b2, FCopy{}, {b}, {o});
        pointwise(FDiffSq{}, {b, PIO2}, {}, 30 + 2 * c);
        MLQ_CUDA(cudaEventRecord(used[c & 1], stream));
    }
    fetch_results();
    ev_give(used[0]);
    ev_give(used[1]);
    ev_give(loaded);
    double out = 0, tot = 0;
    for (int c = 0; c < 3; ++c) {
        out += h_results[30 + 2 * c];
        tot += h_results[31 + 2 * c];
    }
    if (std::isnan(out) || std::isnan(tot)) return std::nan("");
    return tot > 0 ? out / tot : 0.0;
}

// A vector field out: the inverse transform of component c + 1 runs on the
// engine's stream while component c is copied out on the copy stream.
template <typename T>
void Engine<T>::store_vec(const SVec* spec, double* host, int spec_f64) {
    const long nc = spec_ncomp();
    if (spec_f64 < 0) spec_f64 = sf64();
    const int bufs[2] = {PIO, PIO3};
    cudaStream_t xs = slab_ ? nullptr : copy_stream();
    cudaEvent_t done[3] = {ev_take(), ev_take(), ev_take()};
    auto out = [&](int c) {
        if (xs) MLQ_CUDA(cudaStreamWaitEvent(xs, done[c], 0));
        store_scalar_phys(slab_ ? PIO : bufs[c & 1], host + c * n3, xs);  // returns when the copy is done
    };
    for (int c = 0; c < 3; ++c) {
        // the buffer of component c - 2 was copied out by the time out(c - 2) returned
        InvOut o;
        o.nsrc = 1;
        o.src[0] = ZSrc{(const char*)spec + (size_t)c * nc * (spec_f64 ? sizeof(double2) : sizeof(float2)), spec_f64,
                        SYM_ONE, 0, 1.0};
        o.phys_out = slab_ ? PIO : bufs[c & 1];
        inv(b2, {o});
        MLQ_CUDA(cudaEventRecord(done[c], stream));
        if (slab_)
            out(c);
        else if (c >= 1)
            out(c - 1);
    }
    if (!slab_) out(2);
    for (auto e : done) ev_give(e);
}

// ----------------------------------------------------------------------------
// fftwfunction.f90 API on the full band (FP64 engines only)
// ----------------------------------------------------------------------------
template <typename T>
void Engine<T>::fft_c2c(const double* in, double* out, int sign) {
    if (sizeof(T) != 8) throw CudaError("fft API runs in FP64", MLQ_ERR_BADARG);
    const size_t bytes_c = (size_t)n3 * sizeof(cpx<double>);
    cpx<double>* a = (cpx<double>*)dev_alloc(bytes_c);
    cpx<double>* bbuf = (cpx<double>*)dev_alloc(bytes_c);
    try {
        double* st = (double*)stage(bytes_c);
        std::memcpy(st, in, bytes_c);
        MLQ_CUDA(cudaMemcpyAsync(a, st, bytes_c, cudaMemcpyHostToDevice, stream));
        const double scale = sign < 0 ? 1.0 : 1.0 / (double)n3;
        const Band full = make_band(n / 2);
        Band bx = full;  // full complex columns along x
        // x pass: a -> bbuf
        XC2CArgs<double> xa;
        xa.n = n;
        int lx = 8;
        while (lx > 1 && ((size_t)2 * n * lx * sizeof(cpx<double>) > 96 * 1024 || ((long)n * n) % lx != 0)) lx /= 2;
        xa.lx = lx;
        xa.in = a;
        xa.out = bbuf;
        xa.plan = plan(n);
        xa.tw = d_tw;
        xa.scale = 1.0;
        const size_t xsm = (size_t)2 * n * lx * sizeof(cpx<double>);
        if (sign < 0) {
            allow_smem(xc2c_kernel<-1, double>);
            xc2c_kernel<-1, double><<<(unsigned)(((long)n * n) / lx), 256, xsm, stream>>>(xa);
        } else {
            allow_smem(xc2c_kernel<+1, double>);
            xc2c_kernel<+1, double><<<(unsigned)(((long)n * n) / lx), 256, xsm, stream>>>(xa);
        }
        launched();
        // y pass over all n columns: bbuf -> a (full band = natural order)
        const int tx = tx_for();
        YArgs<double> ya;
        ya.n = n;
        ya.nx = n;
        ya.tx = tx;
        ya.band = full;
        ya.in[0] = reinterpret_cast<cpx<double>*>(bbuf);
        ya.out[0] = reinterpret_cast<cpx<double>*>(a);
        ya.plan = plan(n);
        ya.tw = d_tw;
        const size_t ysm = (size_t)2 * n * tx * sizeof(cpx<double>);
        dim3 yg((n + tx - 1) / tx, n, 1);
        if (sign < 0) {
            allow_smem(ypass_kernel<-1, double>);
            ypass_kernel<-1, double><<<yg, 256, ysm, stream>>>(ya);
        } else {
            allow_smem(ypass_kernel<+1, double>);
            ypass_kernel<+1, double><<<yg, 256, ysm, stream>>>(ya);
        }
        launched();
        // z pass: a -> bbuf
        if (sign < 0) {
            ZFwdArgs<double> za;
            za.n = n;
            za.nx = n;
            za.tx = tx;
            za.band = full;
            ZFwdOp op = {};
            op.in = a;
            op.spec_out = bbuf;
            op.spec_f64 = 1;
            op.sym = SYM_ONE;
            op.red_self = -1;
            for (int r = 0; r < 3; ++r) op.red_with_slot[r] = -1;
            za.op[0] = op;
            za.plan = plan(n);
            za.tw = d_tw;
            za.norm = 1.0;
            dim3 zg((n + tx - 1) / tx, n, 1);
            ensure_partials((long)zg.x * zg.y * MAX_RED);
            za.partials = d_partials;
            allow_smem(zfwd_kernel<double>);
            zfwd_kernel<double><<<zg, 256, ysm, stream>>>(za);
        } else {
            ZInvArgs<double> za;
            za.n = n;
            za.nx = n;
            za.tx = tx;
            za.band = full;
            ZInvOp op = {};
            op.src[0] = ZSrc{a, 1, SYM_ONE, 0, scale};
            op.nsrc = 1;
            op.ys_out = bbuf;
            za.op[0] = op;
            za.plan = plan(n);
            za.tw = d_tw;
            dim3 zg((n + tx - 1) / tx, n, 1);
            allow_smem(zinv_kernel<double>);
            zinv_kernel<double><<<zg, 256, ysm, stream>>>(za);
        }
        launched();
        (void)bx;
        MLQ_CUDA(cudaMemcpyAsync(st, bbuf, bytes_c, cudaMemcpyDeviceToHost, stream));
        MLQ_CUDA(cudaStreamSynchronize(stream));
        std::memcpy(out, st, bytes_c);
    } catch (...) {
        free_dev(a);
        free_dev(bbuf);
        throw;
    }
    free_dev(a);
    free_dev(bbuf);
}

template <typename T>
void Engine<T>::fft_r2c(const double* in, double* out) {
    if (sizeof(T) != 8) throw CudaError("fft API runs in FP64", MLQ_ERR_BADARG);
    const Band full = make_band(n / 2);
    widen_to(full);
    load_scalar_phys(in, PIO);
    const size_t nspec = (size_t)full.nb * full.nb * full.nx;
    cpx<double>* sp = (cpx<double>*)dev_alloc(nspec * sizeof(cpx<double>));
    FwdOut o;
    o.spec = sp;
    o.spec_f64 = 1;
    fwd(full, FCopy{}, {PIO}, {o}, -1, -1, 1.0);  // unnormalised like fftfwdr
    double* st = (double*)stage(nspec * sizeof(cpx<double>));
    MLQ_CUDA(cudaMemcpyAsync(st, sp, nspec * sizeof(cpx<double>), cudaMemcpyDeviceToHost, stream));
    MLQ_CUDA(cudaStreamSynchronize(stream));
    std::memcpy(out, st, nspec * sizeof(cpx<double>));
    free_dev(sp);
}

template <typename T>
void Engine<T>::fft_c2r(const double* in, double* out) {
    if (sizeof(T) != 8) throw CudaError("fft API runs in FP64", MLQ_ERR_BADARG);
    const Band full = make_band(n / 2);
    widen_to(full);
    const size_t nspec = (size_t)full.nb * full.nb * full.nx;
    cpx<double>* sp = (cpx<double>*)dev_alloc(nspec * sizeof(cpx<double>));
    double* st = (double*)stage(nspec * sizeof(cpx<double>));
    std::memcpy(st, in, nspec * sizeof(cpx<double>));
    MLQ_CUDA(cudaMemcpyAsync(sp, st, nspec * sizeof(cpx<double>), cudaMemcpyHostToDevice, stream));
    InvOut o;
    o.nsrc = 1;
    o.src[0] = ZSrc{sp, 1, SYM_ONE, 0, 1.0 / (double)n3};  // fftbwdr scales by 1/N^3 (160)
    o.phys_out = PIO;
    inv(full, {o});
    store_scalar_phys(PIO, out);
    free_dev(sp);
}

template <typename T>
void Engine<T>::dealias_scalar(double* g, double order) {
    if (!std::isfinite(order)) throw CudaError("dealias order must be finite", MLQ_ERR_BADARG);
    const int c = band_cut_for_order(n, order);
    if (c < 0) throw CudaError("dealias order < -1 keeps no mode; dealias orders are >= 0", MLQ_ERR_BADARG);
    if (c >= n / 2) return;  // the mask removes nothing (order <= 1)
    const Band bk = make_band(c);
    widen_to(bk);
    load_scalar_phys(g, PIO);
    FwdOut o;
    o.phys_out = PIO2;
    fwd(bk, FCopy{}, {PIO}, {o});
    store_scalar_phys(PIO2, g);
}

template <typename T>
void Engine<T>::widen_to(const Band& b) {
    if (nxcap >= b.nx && nbcap >= b.nb) return;
    for (auto& p : xs_)
        if (p) {
            free_dev(p);
            p = nullptr;
        }
    for (auto& p : ys_)
        if (p) {
            free_dev(p);
            p = nullptr;
        }
    // slab-mode storage is sized by the caps too (slot contents are dropped:
    // callers widen before a pipeline, never between its steps)
    for (auto* v : {&slot_ys_, &xslab_, &slot_pool_})
        for (auto& p : *v)
            if (p) {
                free_dev(p);
                p = nullptr;
            }
    slot_pool_.clear();
    for (auto& sl : slot_)
        if (sl.kind == PSlot::YS) sl.kind = PSlot::NONE;
    nxcap = std::max(nxcap, b.nx);
    nbcap = std::max(nbcap, b.nb);
}

// Fourier coefficients of a host scalar on the full band (FP64 work spectrum)
template <typename T>
static cpx<double>* full_spectrum(Engine<T>& e, const double* host, int phys_idx) {
    const Band full = e.make_band(e.n / 2);
    e.widen_to(full);
    e.load_scalar_phys(host, phys_idx);
    const size_t nspec = (size_t)full.nb * full.nb * full.nx;
    cpx<double>* sp = (cpx<double>*)e.dev_alloc(nspec * sizeof(cpx<double>));
    typename Engine<T>::FwdOut o;
    o.spec = sp;
    o.spec_f64 = 1;
    e.fwd(full, FCopy{}, {phys_idx}, {o});
    return sp;
}

template <typename T>
void Engine<T>::gradient_full(const double* f, double* grad) {
    if (sizeof(T) != 8) throw CudaError("full-band operators run in FP64", MLQ_ERR_BADARG);
    const Band full = make_band(n / 2);
    cpx<double>* sp = full_spectrum(*this, f, PIO);
    for (int j = 0; j < 3; ++j) {
        InvOut o;
        o.nsrc = 1;
        o.src[0] = ZSrc{sp, 1, SYM_IKX + j, 0, 1.0};
        o.phys_out = PIO2;
        inv(full, {o});
        store_scalar_phys(PIO2, grad + j * n3);
    }
    free_dev(sp);
}

template <typename T>
void Engine<T>::divergence_full(const double* u, double* div) {
    if (sizeof(T) != 8) throw CudaError("full-band operators run in FP64", MLQ_ERR_BADARG);
    const Band full = make_band(n / 2);
    cpx<double>* sp[3];
    for (int c = 0; c < 3; ++c) sp[c] = full_spectrum(*this, u + c * n3, PIO);
    InvOut o;
    o.nsrc = 3;
    for (int c = 0; c < 3; ++c) o.src[c] = ZSrc{sp[c], 1, SYM_IKX + c, 0, 1.0};
    o.phys_out = PIO2;
    inv(full, {o});
    store_scalar_phys(PIO2, div);
    for (int c = 0; c < 3; ++c) free_dev(sp[c]);
}

template <typename T>
void Engine<T>::laplacian_full(double* u) {
    if (sizeof(T) != 8) throw CudaError("full-band operators run in FP64", MLQ_ERR_BADARG);
    const Band full = make_band(n / 2);
    for (int c = 0; c < 3; ++c) {
        cpx<double>* sp = full_spectrum(*this, u + c * n3, PIO);
        InvOut o;
        o.nsrc = 1;
        o.src[0] = ZSrc{sp, 1, SYM_NEG_KSQ, 0, 1.0};
        o.phys_out = PIO2;
        inv(full, {o});
        store_scalar_phys(PIO2, u + c * n3);
        free_dev(sp);
    }
}

template <typename T>
void Engine<T>::poisson_full(const double* f, double l, double* phi) {
    if (sizeof(T) != 8) throw CudaError("full-band operators run in FP64", MLQ_ERR_BADARG);
    const Band full = make_band(n / 2);
    cpx<double>* sp = full_spectrum(*this, f, PIO);
    InvOut o;
    o.nsrc = 1;
    o.src[0] = ZSrc{sp, 1, SYM_NEG_INV_KSQ, 0, 1.0 / std::pow(l, 2.0)};  // -f_hat/(l^2 ksq), k=0 -> 0
    o.phys_out = PIO2;
    inv(full, {o});
    store_scalar_phys(PIO2, phi);
    free_dev(sp);
}

// ---- kappa_test_pert (function_ops.f90:615-977) ---------------------------
// The random fields of create-random-poly-b and save-random come from a
// seeded counter generator (the reference draws them from an unseeded
// random_number, 784-785): element i of phi_pert(x,y,z,c) is
// 2 U(seed, i) - 1, U the top 53 bits of the splitmix64 finaliser of
// seed + (i + 1) * 0x9E3779B97F4A7C15.
__device__ __forceinline__ double pert_uniform(unsigned long long seed, long i) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

template <typename T>
__global__ void pert_random_kernel(long n3, unsigned long long seed, T* u0, T* u1, T* u2) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n3; i += (long)gridDim.x * blockDim.x) {
        const int c = (int)(i / n3);
        T* u = c == 0 ? u0 : (c == 1 ? u1 : u2);
        u[i - (long)c * n3] = (T)(2.0 * pert_uniform(seed, i) - 1.0);
    }
}

// "sine" / "divfree-sine" (658-688): m2 is m1 + m3 for the latter
template <typename T>
__global__ void pert_sine_kernel(int n, double m1, double m2, double m3, T* u0, T* u1, T* u2) {
    const long n3 = (long)n * n * n;
    const double PI = 3.14159265358979311600;  // 4 atan2(1, 1)
    const double dx = 1.0 / (double)n;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((long)n * n));
        const double X = (double)x * dx, Y = (double)y * dx, Z = (double)z * dx;
        const double a = 2.0 * PI * m1 * X, b = 2.0 * PI * m2 * Y, c = 2.0 * PI * m3 * Z;
        u0[i] = (T)(sin(a) * cos(b) * cos(c));
        u1[i] = (T)(-cos(a) * sin(b) * cos(c));
        u2[i] = (T)(cos(a) * cos(b) * sin(c));
    }
}

// One spectral pass over the three full-band spectra of a perturbation:
// times scale * f(|K|) (0 at |K| < MACH_EPSILON) when filter > 0 -- 1: m1
// (load-k-random), 2: 10^m2 (|K| / (N/4))^m1 (poly), 3: 10^(-|K|/5) (exp),
// 4: 1 (the k = 0 mode removed) -- then, when leray, divAvg_free
// (2843-2918): u - K_odd (K_odd . u) / |K|^2 with the mean removed (the
// divergence and the gradient each pass through REAL(c2c), which cancels a
// Nyquist index's odd factor; |K|^2 keeps it).
static __global__ void pert_spec_kernel(int n, int nb, int nx, cpx<double>* s0, cpx<double>* s1, cpx<double>* s2, int filter,
                                 double m1, double m2, double scale, int leray) {
    const long ns = (long)nb * nb * nx;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += (long)gridDim.x * blockDim.x) {
        const int fx = (int)(i % nx), fy = (int)((i / nx) % nb), fz = (int)(i / ((long)nx * nb));
        const Kvec k = make_k(n, fx, fy, fz);
        cpx<double> v[3] = {s0[i], s1[i], s2[i]};
        if (filter > 0) {
            const double norm_K = sqrt(k.kx * k.kx + k.ky * k.ky + k.kz * k.kz);
            double f = 0.0;
            if (!(norm_K < MACH_EPSILON)) {
                if (filter == 1)
                    f = m1;
                else if (filter == 2)
                    f = pow(10.0, m2) * pow(norm_K / ((double)n / 4.0), m1);
                else if (filter == 3)
                    f = pow(10.0, -norm_K / 5.0);
                else
                    f = 1.0;
            }
            f *= scale;
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] = v[c] * f;
        }
        if (leray) {
            if (k.ksq > MACH_EPSILON) {
                const cpx<double> d = v[0] * k.ox + v[1] * k.oy + v[2] * k.oz;
                v[0] = v[0] - d * (k.ox / k.ksq);
                v[1] = v[1] - d * (k.oy / k.ksq);
                v[2] = v[2] - d * (k.oz / k.ksq);
            } else {
                v[0] = v[1] = v[2] = mk(0.0, 0.0);
            }
        }
        s0[i] = v[0];
        s1[i] = v[1];
        s2[i] = v[2];
    }
}

template <typename T>
int Engine<T>::kappa_pert(const char* type, double m1, double m2, double m3, const double* loaded,
                          unsigned long long seed, double* out) {
    if (sizeof(T) != 8) throw CudaError("full-band operators run in FP64", MLQ_ERR_BADARG);
    if (!type) throw CudaError("kappa_test_pert: no type", MLQ_ERR_BADARG);
    const std::string t(type);
    enum { SINE, DFSINE, RAW, DIV, SMOOTH_DIV, SMOOTH, KRAND, POLY, EXPF, CREATE, SAVE };
    static const std::map<std::string, int> kinds = {
        {"sine", SINE},
        {"divfree-sine", DFSINE},
        {"load-te0080", RAW},
        {"load-random-a", DIV},
        {"load-random-b", DIV},
        {"load-random-smooth-a", SMOOTH_DIV},
        {"load-random-smooth-b", SMOOTH},
        {"load-k-random-a", KRAND},
        {"load-k-random-b", KRAND},
        {"load-random-poly-a", POLY},
        {"load-random-poly-b", POLY},
        {"load-random-exp-a", EXPF},
        {"load-random-exp-b", EXPF},
        {"create-random-poly-b", CREATE},
        {"save-random", SAVE},
    };
    const auto it = kinds.find(t);
    if (it == kinds.end()) throw CudaError("kappa_test_pert: unknown type " + t, MLQ_ERR_BADARG);
    const int kind = it->second;
    const Band full = make_band(n / 2);
    widen_to(full);
    T* u[3] = {phys(PU), phys(PU + 1), phys(PU + 2)};
    int status = 0;
    // the field
    if (kind == SINE || kind == DFSINE) {
        pert_sine_kernel<T><<<grid_for(n3, 256), 256, 0, stream>>>(n, m1, kind == DFSINE ? m1 + m3 : m2, m3, u[0],
                                                                     u[1], u[2]);
        launched();
    } else if (kind == CREATE || kind == SAVE) {
        pert_random_kernel<T><<<grid_for(3 * n3, 256), 256, 0, stream>>>(n3, seed, u[0], u[1], u[2]);
        launched();
    } else if (loaded) {
        for (int c = 0; c < 3; ++c) load_scalar_phys(loaded + c * n3, PU + c);
    } else {
        for (int c = 0; c < 3; ++c) MLQ_CUDA(cudaMemsetAsync(u[c], 0, n3 * sizeof(T), stream));
        status = 1;
    }
    for (int c = 0; c < 3; ++c) phys_written(PU + c);
    // spectral passes: forward (normalised), the per-mode multiplier and/or
    // divAvg_free, inverse
    const size_t nspec = (size_t)full.nb * full.nb * full.nx;
    cpx<double>* sp[3] = {nullptr, nullptr, nullptr};
    auto spec_pass = [&](int filter, double scale, int leray) {
        for (int c = 0; c < 3; ++c) {
            if (!sp[c]) sp[c] = (cpx<double>*)dev_alloc(nspec * sizeof(cpx<double>));
            FwdOut o;
            o.spec = sp[c];
            o.spec_f64 = 1;
            fwd(full, FCopy{}, {PU + c}, {o});
        }
        pert_spec_kernel<<<grid_for((long)nspec, 256), 256, 0, stream>>>(n, full.nb, full.nx, sp[0], sp[1], sp[2],
                                                                         filter, m1, m2, scale, leray);
        launched();
        for (int c = 0; c < 3; ++c) {
            InvOut o;
            o.nsrc = 1;
            o.src[0] = ZSrc{sp[c], 1, SYM_ONE, 0, 1.0};
            o.phys_out = PU + c;
            inv(full, {o});
        }
    };
    // 100 <phi, phi>_L2 (global_summed_field_inner_product, 3557-3577); a
    // pointwise reduction is already the sum times dV = 1/N^3
    auto norm_const = [&] {
        for (int c = 0; c < 3; ++c) pointwise(FSqRed{}, {PU + c}, {}, 20 + c);
        fetch_results();
        double s = 0.0;
        for (int c = 0; c < 3; ++c) s = s + h_results[20 + c];
        return 100.0 * s;
    };
    try {
        switch (kind) {
            case SINE:
            case DIV: spec_pass(0, 1.0, 1); break;
            case SMOOTH:
            case SMOOTH_DIV: {
                // dealias_scalar(phi(:,:,:,c), 20.0) (708-710): a round trip through
                // the band of order 20
                const int cut = band_cut_for_order(n, 20.0);
                if (cut < n / 2) {
                    const Band bk = make_band(cut);
                    for (int c = 0; c < 3; ++c) {
                        FwdOut o;
                        o.phys_out = PV + c;
                        fwd(bk, FCopy{}, {PU + c}, {o});
                        MLQ_CUDA(cudaMemcpyAsync(u[c], phys(PV + c), n3 * sizeof(T), cudaMemcpyDeviceToDevice, stream));
                    }
                }
                if (kind == SMOOTH_DIV) spec_pass(0, 1.0, 1);
                break;
            }
            case KRAND: spec_pass(1, 1.0, 1); break;
            case POLY: spec_pass(2, 1.0, 1); break;
            case EXPF: spec_pass(3, 1.0, 1); break;
            case CREATE:
            case SAVE: {
                spec_pass(4, 1.0, 1);
                const double nc = norm_const();
                if (kind == CREATE)
                    spec_pass(2, 1.0 / nc, 1);
                else
                    spec_pass(4, 1.0 / nc, 0);  // phi / nc (the field has no k = 0 mode left)
                break;
            }
            default: break;
        }
        for (int c = 0; c < 3; ++c) store_scalar_phys(PU + c, out + c * n3);
    } catch (...) {
        for (auto* p : sp)
            if (p) free_dev(p);
        throw;
    }
    for (auto* p : sp)
        if (p) free_dev(p);
    return status;
}

}  // namespace mlq
