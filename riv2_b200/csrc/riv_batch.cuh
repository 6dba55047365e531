// riv_batch.cuh -- multi-clip (batched) launches of the P-frame encoder's stages.
//
// Included by riv_kernels.cu inside namespace riv (it uses that file's device functions).
// One step of a batch encodes one frame of every clip that has one; each stage below is ONE
// launch over all of them.  A stage's grid is the concatenation of per-clip CTA ranges
// (batch_ctas: prefix sums in BatchLaunch::start), so each CTA works for exactly one clip and
// runs the same per-MB / per-tile device code as the single-clip kernels: the results are those
// of a single-clip encode of the clip, bit for bit.
//
// The search is one cooperative launch whose grid is the concatenation of per-clip wavefront
// launches (SearchParams::cta0 = the clip's first CTA): each clip's row CTAs take its MB rows
// with a stride of its CTA count and wait only on rows of the same clip, all co-resident.

// The clip owning CTA b: the largest c with start[c] <= b (start holds n + 1 prefix sums).
__device__ __forceinline__ int batch_clip(const int* __restrict__ start, int n, int b) {
    int lo = 0, hi = n;  // start[lo] <= b < start[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(start + mid) <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}

__host__ __device__ inline int batch_deblock_tiles(int W, int H, int tw) {
    const int ty = (H / 16) * ((W + tw - 1) / tw);
    const int tc = ((H / 2) / 8) * ((W / 2 + tw / 2 - 1) / (tw / 2));
    return ty + 2 * tc;
}

// CTAs of clip k in stage s (host and device agree through this one function).
__host__ __device__ inline int batch_ctas(int s, const BatchClip& k, const BatchTune& t) {
    const int nmb = k.NMB;
    switch (s) {
        case BS_CONVERT: return k.rgb != nullptr ? ((k.W / 2) * (k.H / 2) + 127) / 128 : 0;
        case BS_TABLE: return k.intra || k.tab == nullptr ? 0 : nmb;
        case BS_PREDICT: return k.intra ? 0 : nmb;
        case BS_AQSUM: return k.intra ? 0 : 1;
        case BS_RESIDUAL: return (nmb + t.res_mbs - 1) / t.res_mbs;
        case BS_DEBLOCK: return k.db_level > 0 ? batch_deblock_tiles(k.W, k.H, t.db_tw) : 0;
        case BS_SCAN: return 1;
        case BS_PACK: return (nmb + 7) / 8;
        default: return 0;
    }
}

// ---- conversion: RGB24 (display size) -> planar YUV 4:2:0, one thread per 2x2 quad
__global__ void __launch_bounds__(128) kb_convert(BatchLaunch b) {
    const int* st = b.start + BS_CONVERT * (b.nclips + 1);
    const int c = batch_clip(st, b.nclips, blockIdx.x);
    const BatchClip& k = b.clips[c];
    const int W = k.W, H = k.H, cw = W / 2, nq = cw * (H / 2);
    const int q = ((int)blockIdx.x - st[c]) * 128 + (int)threadIdx.x;
    if (q >= nq) return;
    uint8_t* Y = k.cur;
    uint8_t* U = Y + (size_t)W * H;
    uint8_t* V = U + (size_t)cw * (H / 2);
    rgb_to_yuv_quad(k.rgb, k.dw, k.dh, Y, U, V, W, q % cw, q / cw);
}

// ---- exhaustive integer SAD table of every P-frame MB (sad_table_mb)
__global__ void __launch_bounds__(128) kb_table(BatchLaunch b) {
    extern __shared__ __align__(16) uint8_t sm[];
    const int* st = b.start + BS_TABLE * (b.nclips + 1);
    const int c = batch_clip(st, b.nclips, blockIdx.x);
    const BatchClip& k = b.clips[c];
    sad_table_mb(k.ref, k.cur, k.W, k.H, k.BW, k.sr, k.tab, k.tstride, (int)blockIdx.x - st[c], sm, threadIdx.x,
                 blockDim.x, 0);
}

// ---- motion-compensated prediction (predict_mb), then the MB's luma variance and its
// glibc-exact ln (k_aq_log's arithmetic) for the AQ mean
__global__ void __launch_bounds__(256) kb_predict(BatchLaunch b) {
    __shared__ unsigned ws[8], ws2[8];
    const int* st = b.start + BS_PREDICT * (b.nclips + 1);
    const int c = batch_clip(st, b.nclips, blockIdx.x);
    const BatchClip& k = b.clips[c];
    const int mb = (int)blockIdx.x - st[c];
    const uint2 vs = predict_mb(k.ref, k.mbo, k.pred, k.W, k.H, mb, ws, ws2);
    if (threadIdx.x == 0) {
        const unsigned long long N = 256ull * vs.y - (unsigned long long)vs.x * vs.x;
        float var = __fdiv_rn(__ull2float_rn(N), 65536.0f);
        var = var < 4.0f ? 4.0f : var;
        k.lnv[mb] = glibc_logf(var, k.logfix, k.nlog);
    }
}

// ---- the strictly sequential mean of a clip's ln variances (aq_sum_cta), one CTA per clip
__global__ void __launch_bounds__(1024) kb_aqsum(BatchLaunch b) {
    extern __shared__ float sl[];
    const int* st = b.start + BS_AQSUM * (b.nclips + 1);
    const BatchClip& k = b.clips[batch_clip(st, b.nclips, blockIdx.x)];
    aq_sum_cta(k.lnv, k.NMB, k.lnv + k.NMB, sl);
}

// ---- residual, transforms, quantisation and reconstruction (residual_mb), NM MBs per CTA
template <int NM>
__global__ void __launch_bounds__(64 * NM) kb_residual(BatchLaunch b) {
    __shared__ __align__(16) int32_t sT16[256], sT16t[256], sT8[64];
    __shared__ __align__(16) ResSmem S[NM];
    const int tid = threadIdx.x;
    for (int i = tid; i < 256; i += 64 * NM) {
        sT16[i] = c_T16[i];
        sT16t[(i & 15) * 16 + (i >> 4)] = c_T16[i];
    }
    if (tid < 64) sT8[tid] = c_T8[tid];
    __syncthreads();
    const int* st = b.start + BS_RESIDUAL * (b.nclips + 1);
    const int c = batch_clip(st, b.nclips, blockIdx.x);
    const BatchClip& k = b.clips[c];
    const int g = tid >> 6, u = tid & 63;
    const int mb = ((int)blockIdx.x - st[c]) * NM + g;
    if (mb >= k.NMB) return;
    residual_mb(k.rp, k.NMB, mb, u, g + 1, S[g], sT16, sT16t, sT8);
}

// ---- out-of-place deblock (deblock_tile), TW luma columns per tile
template <int TW>
__global__ void __launch_bounds__(128) kb_deblock(BatchLaunch b) {
    __shared__ __align__(16) uint8_t tile[(16 + 8) * (TW + 8)];
    const int* st = b.start + BS_DEBLOCK * (b.nclips + 1);
    const int c = batch_clip(st, b.nclips, blockIdx.x);
    const BatchClip& k = b.clips[c];
    const int ty = (k.H / 16) * ((k.W + TW - 1) / TW);
    int t = (int)blockIdx.x - st[c];
    const int plane = t < ty ? 0 : (t - ty) % 2 + 1;
    if (plane > 0) t = (t - ty) / 2;
    deblock_tile<TW>(k.db_src, k.db_dst, k.W, k.H, k.BW, k.db_E, k.db_I, k.db_H, k.db_mask, plane, t, tile, threadIdx.x,
                     blockDim.x, 0);
}

// ---- compaction: the scan (one CTA per clip; it also copies the clip's status word to the
// mapped header, so no separate copy is needed), then one warp per MB
__global__ void __launch_bounds__(SC_THREADS) kb_scan(BatchLaunch b) {
    __shared__ int wsum[SC_THREADS / 32], wsz[SC_THREADS / 32];
    const int* st = b.start + BS_SCAN * (b.nclips + 1);
    const BatchClip& k = b.clips[batch_clip(st, b.nclips, blockIdx.x)];
    scan_mbs<SC_THREADS, SC_IPT>(k.rp.opt_skip, k.rp.eobs, k.NMB, k.intra, k.c_index, k.c_offset, k.c_hdr, threadIdx.x,
                                 1, wsum, wsz);
    if (threadIdx.x == 0) k.c_hdr[2] = *(volatile const unsigned*)k.status;
}
__global__ void __launch_bounds__(256) kb_pack(BatchLaunch b) {
    const int* st = b.start + BS_PACK * (b.nclips + 1);
    const int c = batch_clip(st, b.nclips, blockIdx.x);
    const BatchClip& k = b.clips[c];
    const int m = ((int)blockIdx.x - st[c]) * 8 + (threadIdx.x >> 5);
    if (m < k.NMB)
        pack_mb(m, threadIdx.x & 31, k.rp.opt_skip, k.rp.mb, k.rp.coeffs, k.rp.eobs, k.c_index, k.c_offset, k.intra,
                k.c_side, k.c_packed, k.c_peobs);
}

// ---- the multi-clip search wavefront (per-MB reference windows; see the file comment)
template <bool TABLE, bool SMALL>
__global__ void __maxnreg__(120) k_search_multi(const SearchParams* __restrict__ ps, const int* __restrict__ start,
                                                int nclips) {
    search_body<false, TABLE, SMALL>(ps[batch_clip(start, nclips, blockIdx.x)]);
}

static const void* search_multi_fn(bool table, bool small) {
    if (table && small) return (const void*)k_search_multi<true, true>;
    if (table) return (const void*)k_search_multi<true, false>;
    return (const void*)k_search_multi<false, false>;
}

static size_t batch_stage_smem(int s, int max_sr) {
    if (s == BS_TABLE) return sad_table_smem(max_sr);
    if (s == BS_AQSUM) return 8192 * sizeof(float);
    return 0;
}

static int batch_stage_threads(int s, const BatchTune& t) {
    switch (s) {
        case BS_CONVERT: case BS_TABLE: case BS_DEBLOCK: return 128;
        case BS_PREDICT: case BS_PACK: return 256;
        case BS_AQSUM: return 1024;
        case BS_RESIDUAL: return 64 * t.res_mbs;
        case BS_SCAN: return SC_THREADS;
        default: return 0;
    }
}

int batch_ctas_host(int s, const BatchClip& k, const BatchTune& t) { return batch_ctas(s, k, t); }

int launch_batch_stage(int s, const BatchLaunch& b, const BatchTune& t, int total, int max_sr, void* stream) {
    if (total <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t sm = batch_stage_smem(s, max_sr);
    const int nt = batch_stage_threads(s, t);
    switch (s) {
        case BS_CONVERT: kb_convert<<<total, nt, 0, st>>>(b); break;
        case BS_TABLE:
            if (sm > 48 * 1024) {
                cudaError_t e = cudaFuncSetAttribute(kb_table, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                if (e != cudaSuccess) return (int)e;
            }
            kb_table<<<total, nt, sm, st>>>(b);
            break;
        case BS_PREDICT: kb_predict<<<total, nt, 0, st>>>(b); break;
        case BS_AQSUM: kb_aqsum<<<total, nt, sm, st>>>(b); break;
        case BS_RESIDUAL:
            if (t.res_mbs == 2) kb_residual<2><<<total, nt, 0, st>>>(b);
            else if (t.res_mbs == 4) kb_residual<4><<<total, nt, 0, st>>>(b);
            else if (t.res_mbs == 8) kb_residual<8><<<total, nt, 0, st>>>(b);
            else return (int)cudaErrorInvalidValue;
            break;
        case BS_DEBLOCK:
            if (t.db_tw == 64) kb_deblock<64><<<total, nt, 0, st>>>(b);
            else if (t.db_tw == 128) kb_deblock<128><<<total, nt, 0, st>>>(b);
            else if (t.db_tw == 256) kb_deblock<256><<<total, nt, 0, st>>>(b);
            else return (int)cudaErrorInvalidValue;
            break;
        case BS_SCAN: kb_scan<<<total, nt, 0, st>>>(b); break;
        case BS_PACK: kb_pack<<<total, nt, 0, st>>>(b); break;
        default: return (int)cudaErrorInvalidValue;
    }
    return (int)cudaGetLastError();
}

int search_multi_capacity(bool table, bool small, int max_sr, int* per_sm, size_t* smem, int* threads) {
    const void* fn = search_multi_fn(table, small);
    const size_t sm = search_smem(max_sr, 0, false, table);
    const int nt = search_threads(false, table);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fn, nt, sm);
    *smem = sm;
    *threads = nt;
    return (int)e;
}

int launch_search_multi(const SearchParams* dparams, const int* dstart, int nclips, int total, bool table, bool small,
                        size_t smem, int threads, void* stream) {
    if (total <= 0) return 0;
    void* args[] = {(void*)&dparams, (void*)&dstart, (void*)&nclips};
    // cooperative: every clip's row CTAs are co-resident, so each row's wait on the row above
    // (a CTA of the same clip) can always make progress
    return (int)cudaLaunchCooperativeKernel(search_multi_fn(table, small), dim3(total), dim3(threads), args, smem,
                                            (cudaStream_t)stream);
}
