// MEX gateway: MATLAB -> libpkdecon.so.  Build inside MATLAB with
//   mex -R2018a pkdecon_mex.cpp -I<repo>/include -L<repo>/petakit5d_b200/lib -lpkdecon
// (mex.h comes with MATLAB; this file is not compiled by the repository's own build).
//
//   J        = pkdecon_mex('omw', I, PSF_f, PSF_b, NUMIT, opts)   % decon_lucy_omw_function
//   [J, k]   = pkdecon_mex('rl', I, PSF, NUMIT, opts)             % decon_lucy_function
//   [b, otf, absc, mask] = pkdecon_mex('omw_bp', psf, alpha, skewed, thresh, area, hann, minInt)
//   [bp, otf] = pkdecon_mex('wb_bp', psf, alpha, beta, n, resFlag, iRes)
//   psf      = pkdecon_mex('psf_gen', psf, dz_psf, dz_data, medFactor, PSFGenMethod)  % psf_gen_new
//   volout   = pkdecon_mex('dsr', vol, angle, dz, xyPixelSize, reverse, objectiveScan, xStepThresh, bbox, save16bit)
//                                                                 % deskewRotateFrame3D
//   J        = pkdecon_mex('edgetaper', vol, PSF)                 % edgetaper of every z slice (RLdecon.m:352-357)
//   mask     = pkdecon_mex('mask_erosion', im, EdgeErosion)       % decon_mask_edge_erosion(im > 0, E)
//   data     = pkdecon_mex('readtiff', path[, [z1 z2]])            % parallelReadTiff
//   pkdecon_mex('writetiff', path, data, compression)             % parallelWriteTiff ('lzw' | 'none')
//   sz       = pkdecon_mex('tiffsize', path)                      % getImageSizeMex
//   data     = pkdecon_mex('readzarr', path[, bbox])               % parallelReadZarr (none / zlib / gzip)
//   pkdecon_mex('writezarr', path, data, blockSize)               % writezarr (order F, zlib)
//   pkdecon_mex('reset')                                           % reset(gpuDevice) analogue
// opts: struct with the reference's name/value fields (Background, save16bit, dampFactor,
// scaleFactor, deconOffset, EdgeErosion, bbox).  Errors are raised with mexErrMsgIdAndTxt using the
// identifier "pkdecon:<status>" and pk_last_error() (the convention of crop3d_mex.c:36-63).
#include <cstring>
#include <vector>
#include <string>

#include "mex.h"
#include "pkdecon.h"

static pk_ctx* g_ctx = nullptr;

static void at_exit() {
    if (g_ctx) pk_ctx_destroy(g_ctx);
    g_ctx = nullptr;
}

static pk_ctx* ctx() {
    if (!g_ctx) {
        g_ctx = pk_ctx_create(0);
        if (!g_ctx) mexErrMsgIdAndTxt("pkdecon:cuda", "%s", pk_last_error());
        mexAtExit(at_exit);
    }
    return g_ctx;
}

static void check(pk_status s) {
    static const char* names[] = {"ok", "invalid", "unsupported", "cuda", "nomem", "busy", "timeout", "cancelled",
                                  "emptyOTFMask"};
    if (s != PK_OK) {
        std::string id = std::string("pkdecon:") + (s >= 0 && s <= 8 ? names[s] : "unknown");
        mexErrMsgIdAndTxt(id.c_str(), "%s", pk_last_error());
    }
}

static void dims3(const mxArray* a, int64_t d[3]) {
    const mwSize nd = mxGetNumberOfDimensions(a);
    const mwSize* s = mxGetDimensions(a);
    if (nd > 3) mexErrMsgIdAndTxt("pkdecon:invalid", "at most 3 dimensions");
    for (int i = 0; i < 3; i++) d[i] = i < (int)nd ? (int64_t)s[i] : 1;
}

static double field(const mxArray* opts, const char* name, double def) {
    if (!opts || !mxIsStruct(opts)) return def;
    const mxArray* f = mxGetField(opts, 0, name);
    if (!f || mxIsEmpty(f)) return def;
    return mxGetScalar(f);
}

static void params(const mxArray* opts, pk_decon_params* p) {
    pk_params_default(p);
    p->background = field(opts, "Background", 0.0);
    p->save16bit = field(opts, "save16bit", 1.0) != 0;
    p->damp_factor = field(opts, "dampFactor", 1.0);
    p->scale_factor = field(opts, "scaleFactor", 1.0);
    p->decon_offset = field(opts, "deconOffset", 0.0);
    p->edge_erosion = (int32_t)field(opts, "EdgeErosion", 0.0);
    const mxArray* bb = opts && mxIsStruct(opts) ? mxGetField(opts, 0, "bbox") : nullptr;
    if (bb && !mxIsEmpty(bb)) {
        if (mxGetNumberOfElements(bb) != 6) mexErrMsgIdAndTxt("pkdecon:invalid", "bbox must have 6 elements");
        const double* v = mxGetPr(bb);
        p->has_bbox = 1;
        for (int i = 0; i < 6; i++) p->bbox[i] = (int64_t)v[i];
    }
}

static pk_dtype dtype_of(const mxArray* a) {
    switch (mxGetClassID(a)) {
        case mxUINT16_CLASS: return PK_U16;
        case mxSINGLE_CLASS: return PK_F32;
        case mxDOUBLE_CLASS: return PK_F64;
        default: mexErrMsgIdAndTxt("pkdecon:invalid", "I must be uint16, single or double");
    }
    return PK_U16;
}

static const float* single_psf(const mxArray* a) {
    if (mxGetClassID(a) != mxSINGLE_CLASS) mexErrMsgIdAndTxt("pkdecon:invalid", "PSFs must be single (use single(psf))");
    return (const float*)mxGetData(a);
}

static mxArray* make_out(const int64_t od[3], bool u16) {
    const mwSize d[3] = {(mwSize)od[0], (mwSize)od[1], (mwSize)od[2]};
    return mxCreateNumericArray(3, d, u16 ? mxUINT16_CLASS : mxSINGLE_CLASS, mxREAL);
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    if (nrhs < 1 || !mxIsChar(prhs[0])) mexErrMsgIdAndTxt("pkdecon:invalid", "first argument: command string");
    char cmd[32];
    mxGetString(prhs[0], cmd, sizeof(cmd));
    if (!strcmp(cmd, "reset")) {
        check(pk_ctx_reset(ctx()));
        return;
    }
    if (!strcmp(cmd, "omw") || !strcmp(cmd, "rl")) {
        const bool omw = !strcmp(cmd, "omw");
        const int base = omw ? 5 : 4;
        if (nrhs < base) mexErrMsgIdAndTxt("pkdecon:invalid", "not enough arguments");
        const mxArray* I = prhs[1];
        int64_t d[3], pf[3], pb[3], od[3];
        dims3(I, d);
        dims3(prhs[2], pf);
        pk_decon_params p;
        params(nrhs > base ? prhs[base] : nullptr, &p);
        pk_output_dims(d, &p, od);
        plhs[0] = make_out(od, p.save16bit != 0);
        if (omw) {
            dims3(prhs[3], pb);
            check(pk_decon_lucy_omw(ctx(), mxGetData(I), dtype_of(I), d, single_psf(prhs[2]), pf, single_psf(prhs[3]),
                                    pb, (int32_t)mxGetScalar(prhs[4]), &p, mxGetData(plhs[0])));
        } else {
            int32_t k = 0;
            check(pk_decon_lucy(ctx(), mxGetData(I), dtype_of(I), d, single_psf(prhs[2]), pf,
                                (int32_t)mxGetScalar(prhs[3]), &p, mxGetData(plhs[0]), &k));
            if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(k);
        }
        return;
    }
    if (!strcmp(cmd, "debug")) {
        // [J, err_mat, snaps] = pkdecon_mex('debug', method, I, PSF_f, PSF_b, NUMIT, opts, saveStep)
        // method 'omw' or 'rl' (PSF_b ignored); snaps = uint16 [ny nx nz nsnap], every saveStep-th J
        if (nrhs < 8 || !mxIsChar(prhs[1])) mexErrMsgIdAndTxt("pkdecon:invalid", "debug: not enough arguments");
        char m[8];
        mxGetString(prhs[1], m, sizeof(m));
        const int32_t method = !strcmp(m, "omw") ? 1 : 0;
        const mxArray* I = prhs[2];
        int64_t d[3], pf[3], pb[3], od[3];
        dims3(I, d);
        dims3(prhs[3], pf);
        if (method == 1) dims3(prhs[4], pb);
        else for (int i = 0; i < 3; i++) pb[i] = pf[i];
        const int32_t numit = (int32_t)mxGetScalar(prhs[5]);
        pk_decon_params p;
        params(prhs[6], &p);
        const int32_t step = (int32_t)mxGetScalar(prhs[7]);
        pk_output_dims(d, &p, od);
        plhs[0] = make_out(od, p.save16bit != 0);
        const int32_t nsnap = step > 0 ? numit / step : 0;
        const mwSize sd[4] = {(mwSize)d[0], (mwSize)d[1], (mwSize)d[2], (mwSize)(nsnap > 0 ? nsnap : 0)};
        mxArray* snaps = mxCreateNumericArray(4, sd, mxUINT16_CLASS, mxREAL);
        std::vector<double> err((size_t)(numit > 0 ? numit : 1) * 4);
        int32_t rows = 0;
        check(pk_decon_debug(ctx(), method, mxGetData(I), dtype_of(I), d, single_psf(prhs[3]), pf,
                             method == 1 ? single_psf(prhs[4]) : nullptr, pb, numit, &p, step, mxGetData(plhs[0]),
                             err.data(), &rows, nsnap > 0 ? (uint16_t*)mxGetData(snaps) : nullptr));
        if (nlhs > 1) {
            plhs[1] = mxCreateDoubleMatrix((mwSize)rows, 4, mxREAL);
            memcpy(mxGetPr(plhs[1]), err.data(), sizeof(double) * (size_t)rows * 4);   // column-major rows x 4
        }
        if (nlhs > 2) plhs[2] = snaps;
        else mxDestroyArray(snaps);
        return;
    }
    if (!strcmp(cmd, "omw_bp")) {
        if (nrhs < 8) mexErrMsgIdAndTxt("pkdecon:invalid", "omw_bp: psf, alpha, skewed, thresh, area, hann, minInt");
        int64_t pd[3];
        dims3(prhs[1], pd);
        const int32_t skewed = mxIsEmpty(prhs[3]) ? -1 : (mxGetScalar(prhs[3]) != 0);
        const double* hann = mxGetPr(prhs[6]);
        const mwSize dd[3] = {(mwSize)pd[0], (mwSize)pd[1], (mwSize)pd[2]};
        plhs[0] = mxCreateNumericArray(3, dd, mxSINGLE_CLASS, mxREAL);
        mxArray* otf = mxCreateNumericArray(3, dd, mxSINGLE_CLASS, mxCOMPLEX);   // interleaved (R2018a API)
        mxArray* absc = mxCreateNumericArray(3, dd, mxSINGLE_CLASS, mxREAL);
        mxArray* mask = mxCreateNumericArray(3, dd, mxUINT8_CLASS, mxREAL);
        check(pk_omw_backprojector(ctx(), single_psf(prhs[1]), pd, mxGetScalar(prhs[2]), skewed, mxGetScalar(prhs[4]),
                                   mxGetScalar(prhs[5]), hann[0], hann[1], mxGetScalar(prhs[7]),
                                   (float*)mxGetData(plhs[0]), (float*)mxGetComplexSingles(otf),
                                   (float*)mxGetData(absc), (uint8_t*)mxGetData(mask)));
        if (nlhs > 1) plhs[1] = otf; else mxDestroyArray(otf);
        if (nlhs > 2) plhs[2] = absc; else mxDestroyArray(absc);
        if (nlhs > 3) plhs[3] = mask; else mxDestroyArray(mask);
        return;
    }
    if (!strcmp(cmd, "wb_bp") || !strcmp(cmd, "bp")) {
        // wb_bp: psf, alpha, beta, n, resFlag[, iRes]; bp: psf, bp_type, alpha, beta, n, resFlag[, iRes]
        const int o = strcmp(cmd, "bp") ? 0 : 1;
        if (nrhs < 6 + o) mexErrMsgIdAndTxt("pkdecon:invalid", "bp: psf, bp_type, alpha, beta, n, resFlag[, iRes]");
        int32_t type = PK_BP_WIENER_BUTTERWORTH;
        if (o) {
            if (!mxIsChar(prhs[2])) mexErrMsgIdAndTxt("pkdecon:invalid", "bp_type must be a string");
            char t[32];
            mxGetString(prhs[2], t, sizeof(t));
            const char* names[] = {"traditional", "gaussian", "butterworth", "wiener", "wiener-butterworth"};
            type = -1;
            for (int i = 0; i < 5; i++)
                if (!strcmp(t, names[i])) type = i;
            if (type < 0) mexErrMsgIdAndTxt("pkdecon:invalid", "bp_type does not match any back-projector type");
        }
        int64_t pd[3];
        dims3(prhs[1], pd);
        double ires[3] = {0, 0, 0};
        if (nrhs > 6 + o && mxGetNumberOfElements(prhs[6 + o]) == 3) memcpy(ires, mxGetPr(prhs[6 + o]), sizeof(ires));
        const mwSize dd[3] = {(mwSize)pd[0], (mwSize)pd[1], (mwSize)pd[2]};
        plhs[0] = mxCreateNumericArray(3, dd, mxDOUBLE_CLASS, mxREAL);
        mxArray* otf = mxCreateNumericArray(3, dd, mxDOUBLE_CLASS, mxCOMPLEX);
        check(pk_backprojector(ctx(), single_psf(prhs[1]), pd, type, mxGetScalar(prhs[2 + o]), mxGetScalar(prhs[3 + o]),
                               (int32_t)mxGetScalar(prhs[4 + o]), (int32_t)mxGetScalar(prhs[5 + o]), ires,
                               mxGetPr(plhs[0]), (double*)mxGetComplexDoubles(otf)));
        if (nlhs > 1) plhs[1] = otf; else mxDestroyArray(otf);
        return;
    }
    if (!strcmp(cmd, "psf_gen")) {
        if (nrhs < 6 || !mxIsChar(prhs[5])) mexErrMsgIdAndTxt("pkdecon:invalid", "psf_gen: psf, dz_psf, dz_data, medFactor, PSFGenMethod");
        int64_t pd[3], od[3];
        dims3(prhs[1], pd);
        char m[16];
        mxGetString(prhs[5], m, sizeof(m));
        int32_t method;
        if (!strcmp(m, "masked")) method = 0;
        else if (!strcmp(m, "median")) method = 1;
        else mexErrMsgIdAndTxt("pkdecon:invalid", "PSFGenMethod must be 'masked' or 'median'");
        const float* psf = single_psf(prhs[1]);
        const double dzp = mxGetScalar(prhs[2]), dzd = mxGetScalar(prhs[3]), mf = mxGetScalar(prhs[4]);
        check(pk_psf_gen(ctx(), psf, pd, dzp, dzd, mf, method, nullptr, 0, od));
        const mwSize dd[3] = {(mwSize)od[0], (mwSize)od[1], (mwSize)od[2]};
        plhs[0] = mxCreateNumericArray(3, dd, mxSINGLE_CLASS, mxREAL);
        check(pk_psf_gen(ctx(), psf, pd, dzp, dzd, mf, method, (float*)mxGetData(plhs[0]), (int64_t)(od[0] * od[1] * od[2]), od));
        return;
    }
    if (!strcmp(cmd, "dsr")) {
        if (nrhs < 10) mexErrMsgIdAndTxt("pkdecon:invalid", "dsr: vol, angle, dz, xyPixelSize, reverse, objectiveScan, xStepThresh, bbox, save16bit");
        int64_t d[3], od[3], bb[6];
        dims3(prhs[1], d);
        pk_dtype t;
        if (mxGetClassID(prhs[1]) == mxUINT16_CLASS) t = PK_U16;
        else if (mxGetClassID(prhs[1]) == mxSINGLE_CLASS) t = PK_F32;
        else mexErrMsgIdAndTxt("pkdecon:invalid", "vol must be uint16 or single");
        const int64_t* pbb = nullptr;
        if (!mxIsEmpty(prhs[8])) {
            if (mxGetNumberOfElements(prhs[8]) != 6) mexErrMsgIdAndTxt("pkdecon:invalid", "bbox must have 6 elements");
            for (int k = 0; k < 6; k++) bb[k] = (int64_t)mxGetPr(prhs[8])[k];
            pbb = bb;
        }
        const double ang = mxGetScalar(prhs[2]), dz = mxGetScalar(prhs[3]), px = mxGetScalar(prhs[4]);
        const int32_t rev = mxGetScalar(prhs[5]) != 0, obj = mxGetScalar(prhs[6]) != 0, s16 = mxGetScalar(prhs[9]) != 0;
        const double thr = mxGetScalar(prhs[7]);
        const void* in = mxGetData(prhs[1]);
        check(pk_deskew_rotate(ctx(), in, t, d, ang, dz, px, rev, obj, thr, pbb, s16, nullptr, od));
        const mwSize dd[3] = {(mwSize)od[0], (mwSize)od[1], (mwSize)od[2]};
        plhs[0] = mxCreateNumericArray(3, dd, (s16 && t == PK_U16) ? mxUINT16_CLASS : mxSINGLE_CLASS, mxREAL);
        check(pk_deskew_rotate(ctx(), in, t, d, ang, dz, px, rev, obj, thr, pbb, s16, mxGetData(plhs[0]), od));
        return;
    }
    if (!strcmp(cmd, "edgetaper")) {
        if (nrhs < 3) mexErrMsgIdAndTxt("pkdecon:invalid", "edgetaper: vol, PSF");
        int64_t d[3], pd[3];
        dims3(prhs[1], d);
        dims3(prhs[2], pd);
        pk_dtype t;
        if (mxGetClassID(prhs[1]) == mxUINT16_CLASS) t = PK_U16;
        else if (mxGetClassID(prhs[1]) == mxSINGLE_CLASS) t = PK_F32;
        else mexErrMsgIdAndTxt("pkdecon:invalid", "vol must be uint16 or single");
        if (mxGetClassID(prhs[2]) != mxDOUBLE_CLASS || pd[2] != 1) mexErrMsgIdAndTxt("pkdecon:invalid", "PSF must be a 2-D double array");
        const mwSize dd[3] = {(mwSize)d[0], (mwSize)d[1], (mwSize)d[2]};
        plhs[0] = mxCreateNumericArray(3, dd, t == PK_U16 ? mxUINT16_CLASS : mxSINGLE_CLASS, mxREAL);
        check(pk_edgetaper(ctx(), mxGetData(prhs[1]), t, d, mxGetPr(prhs[2]), pd, mxGetData(plhs[0])));
        return;
    }
    if (!strcmp(cmd, "mask_erosion")) {
        if (nrhs < 3) mexErrMsgIdAndTxt("pkdecon:invalid", "mask_erosion: im, EdgeErosion");
        int64_t d[3];
        dims3(prhs[1], d);
        pk_dtype t;
        if (mxGetClassID(prhs[1]) == mxUINT16_CLASS) t = PK_U16;
        else if (mxGetClassID(prhs[1]) == mxSINGLE_CLASS) t = PK_F32;
        else mexErrMsgIdAndTxt("pkdecon:invalid", "im must be uint16 or single");
        const mwSize dd[3] = {(mwSize)d[0], (mwSize)d[1], (mwSize)d[2]};
        plhs[0] = mxCreateLogicalArray(3, dd);                                // logical: one byte, 0 or 1
        check(pk_mask_edge_erosion(ctx(), mxGetData(prhs[1]), t, d, (int32_t)mxGetScalar(prhs[2]),
                                   (uint8_t*)mxGetData(plhs[0])));
        return;
    }
    if (!strcmp(cmd, "readtiff") || !strcmp(cmd, "tiffsize")) {
        if (nrhs < 2 || !mxIsChar(prhs[1])) mexErrMsgIdAndTxt("pkdecon:invalid", "%s: file name", cmd);
        std::vector<char> path(mxGetNumberOfElements(prhs[1]) + 1);
        mxGetString(prhs[1], path.data(), (mwSize)path.size());
        int64_t d[3];
        int32_t bits = 0, isf = 0;
        check(pk_tiff_info(path.data(), d, &bits, &isf));
        if (!strcmp(cmd, "tiffsize")) {
            plhs[0] = mxCreateDoubleMatrix(1, 3, mxREAL);
            for (int k = 0; k < 3; k++) mxGetPr(plhs[0])[k] = (double)d[k];
            return;
        }
        int64_t rng[2];
        const int64_t* pr = nullptr;
        if (nrhs > 2 && !mxIsEmpty(prhs[2])) {
            if (mxGetNumberOfElements(prhs[2]) != 2) mexErrMsgIdAndTxt("pkdecon:invalid", "Input range is not 2");
            rng[0] = (int64_t)mxGetPr(prhs[2])[0];
            rng[1] = (int64_t)mxGetPr(prhs[2])[1];
            d[2] = rng[1] - rng[0] + 1;
            pr = rng;
        }
        mxClassID c;
        if (isf) c = bits == 64 ? mxDOUBLE_CLASS : mxSINGLE_CLASS;
        else c = bits == 8 ? mxUINT8_CLASS : bits == 16 ? mxUINT16_CLASS : mxUINT32_CLASS;
        const mwSize dd[3] = {(mwSize)d[0], (mwSize)d[1], (mwSize)(d[2] > 0 ? d[2] : 0)};
        plhs[0] = mxCreateNumericArray(3, dd, c, mxREAL);
        check(pk_tiff_read(path.data(), pr, mxGetData(plhs[0]), (int64_t)(mxGetElementSize(plhs[0]) * mxGetNumberOfElements(plhs[0])), 0));
        return;
    }
    if (!strcmp(cmd, "writetiff")) {
        if (nrhs < 3 || !mxIsChar(prhs[1])) mexErrMsgIdAndTxt("pkdecon:invalid", "writetiff: file name, data[, compression]");
        std::vector<char> path(mxGetNumberOfElements(prhs[1]) + 1);
        mxGetString(prhs[1], path.data(), (mwSize)path.size());
        int32_t bits, isf = 0;
        switch (mxGetClassID(prhs[2])) {
            case mxUINT8_CLASS: case mxLOGICAL_CLASS: bits = 8; break;
            case mxUINT16_CLASS: bits = 16; break;
            case mxUINT32_CLASS: bits = 32; break;
            case mxSINGLE_CLASS: bits = 32; isf = 1; break;
            case mxDOUBLE_CLASS: bits = 64; isf = 1; break;
            default: mexErrMsgIdAndTxt("pkdecon:invalid", "Data type not suppported");
        }
        char comp[8] = "lzw";
        if (nrhs > 3 && mxIsChar(prhs[3])) mxGetString(prhs[3], comp, sizeof(comp));
        int64_t d[3];
        dims3(prhs[2], d);
        check(pk_tiff_write(path.data(), mxGetData(prhs[2]), d, bits, isf, strcmp(comp, "none") != 0, 0));
        return;
    }
    if (!strcmp(cmd, "readzarr")) {
        if (nrhs < 2 || !mxIsChar(prhs[1])) mexErrMsgIdAndTxt("pkdecon:invalid", "readzarr: file name[, bbox]");
        std::vector<char> path(mxGetNumberOfElements(prhs[1]) + 1);
        mxGetString(prhs[1], path.data(), (mwSize)path.size());
        int64_t d[3], ch[3], bb[6];
        int32_t bits = 0, isf = 0;
        check(pk_zarr_info(path.data(), d, ch, &bits, &isf));
        const int64_t* pb = nullptr;
        if (nrhs > 2 && !mxIsEmpty(prhs[2])) {
            if (mxGetNumberOfElements(prhs[2]) != 6) mexErrMsgIdAndTxt("pkdecon:invalid", "bbox must have 6 elements");
            for (int k = 0; k < 6; k++) bb[k] = (int64_t)mxGetPr(prhs[2])[k];
            for (int k = 0; k < 3; k++) d[k] = bb[k + 3] - bb[k] + 1;
            pb = bb;
        }
        mxClassID c;
        if (isf) c = bits == 64 ? mxDOUBLE_CLASS : mxSINGLE_CLASS;
        else c = bits == 8 ? mxUINT8_CLASS : bits == 16 ? mxUINT16_CLASS : mxUINT32_CLASS;
        const mwSize dd[3] = {(mwSize)d[0], (mwSize)d[1], (mwSize)d[2]};
        plhs[0] = mxCreateNumericArray(3, dd, c, mxREAL);
        check(pk_zarr_read(path.data(), pb, mxGetData(plhs[0]), (int64_t)(mxGetElementSize(plhs[0]) * mxGetNumberOfElements(plhs[0])), 0));
        return;
    }
    if (!strcmp(cmd, "writezarr")) {
        if (nrhs < 3 || !mxIsChar(prhs[1])) mexErrMsgIdAndTxt("pkdecon:invalid", "writezarr: file name, data[, blockSize]");
        std::vector<char> path(mxGetNumberOfElements(prhs[1]) + 1);
        mxGetString(prhs[1], path.data(), (mwSize)path.size());
        int32_t bits, isf = 0;
        switch (mxGetClassID(prhs[2])) {
            case mxUINT8_CLASS: case mxLOGICAL_CLASS: bits = 8; break;
            case mxUINT16_CLASS: bits = 16; break;
            case mxUINT32_CLASS: bits = 32; break;
            case mxSINGLE_CLASS: bits = 32; isf = 1; break;
            case mxDOUBLE_CLASS: bits = 64; isf = 1; break;
            default: mexErrMsgIdAndTxt("pkdecon:invalid", "Data type not suppported");
        }
        int64_t d[3], bs[3] = {500, 500, 500};
        dims3(prhs[2], d);
        if (nrhs > 3 && mxGetNumberOfElements(prhs[3]) >= 3)
            for (int k = 0; k < 3; k++) bs[k] = (int64_t)mxGetPr(prhs[3])[k];
        check(pk_zarr_write(path.data(), mxGetData(prhs[2]), d, bits, isf, bs, 1, 0));
        return;
    }
    mexErrMsgIdAndTxt("pkdecon:invalid", "unknown command '%s'", cmd);
}
