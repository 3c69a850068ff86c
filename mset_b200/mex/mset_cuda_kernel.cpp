// mset_cuda_kernel.cpp -- MEX gateway that puts libmset_b200 behind the call
// signature of the reference's CUDA module, so Run_MSET_recon.m calls it
// unchanged:
//
//   mset_cuda_kernel('upload', STEM_data, STEM_data.measured_4D_data);
//   [RVol, probe, x, y(, err)] = mset_cuda_kernel('run_mset' | 'run_sset', STEM_data, cells);
//   err = mset_cuda_kernel('error_mset' | 'error_sset', STEM_data, cells);
//   clear mset_cuda_kernel
//
// Modes, inputs and outputs (classes, shapes, the error normalisation, the
// error message for an unknown mode) are those of src/CUDA/mex_main.cu:19-184.
// Struct fields of any numeric class are read as single, as the reference's
// get_Mxdata does (mex_tools.cpp).  The measured cell is not gathered on the
// host: its patterns go to the library as a pointer table
// (mset_mex_upload_cells), as the reference borrows the cell (mex_main.cu:87).
//
// Build with MATLAB:
//   mex -R2018a mset_cuda_kernel.cpp -I<repo>/include -L<repo>/mset_b200 -lmset_b200
// It uses the MEX functions the reference's own gateway uses, and mxFree.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "mex.h"
#include "mset_b200.h"

namespace {

// STEM_data.<name> of a 1x1 struct
const mxArray *field(const mxArray *s, const char *name) {
    const int nf = mxGetNumberOfFields(s);
    for (int i = 0; i < nf; ++i)
        if (std::strcmp(mxGetFieldNameByNumber(s, i), name) == 0) return mxGetFieldByNumber(s, 0, i);
    std::string msg = std::string("STEM_data has no field '") + name + "'";
    mexErrMsgTxt(msg.c_str());
    return nullptr;
}

// real numeric array of any class as single values
std::vector<float> to_single(const mxArray *a) {
    const size_t n = mxGetNumberOfElements(a);
    std::vector<float> v(n);
    switch (mxGetClassID(a)) {
    case mxSINGLE_CLASS: std::memcpy(v.data(), mxGetSingles(a), sizeof(float) * n); break;
    case mxDOUBLE_CLASS: {
        const double *d = mxGetDoubles(a);
        for (size_t i = 0; i < n; ++i) v[i] = (float)d[i];
        break;
    }
    case mxINT32_CLASS: {
        const int32_t *d = mxGetInt32s(a);
        for (size_t i = 0; i < n; ++i) v[i] = (float)d[i];
        break;
    }
    case mxUINT8_CLASS: {
        const uint8_t *d = mxGetUint8s(a);
        for (size_t i = 0; i < n; ++i) v[i] = (float)d[i];
        break;
    }
    case mxLOGICAL_CLASS: {
        const mxLogical *d = mxGetLogicals(a);
        for (size_t i = 0; i < n; ++i) v[i] = d[i] ? 1.f : 0.f;
        break;
    }
    default: mexErrMsgTxt("numeric input expected");
    }
    return v;
}

float scalar(const mxArray *s, const char *name) {
    const std::vector<float> v = to_single(field(s, name));
    if (v.empty()) mexErrMsgTxt("empty scalar field");
    return v[0];
}

// complex single array, interleaved (re, im)
const float *complex_single(const mxArray *s, const char *name) {
    const mxArray *a = field(s, name);
    if (mxGetClassID(a) != mxSINGLE_CLASS) mexErrMsgTxt("init_wave2D and prop2D must be complex single");
    return reinterpret_cast<const float *>(mxGetComplexSingles(a));
}

mxArray *single_array(mwSize ndim, const mwSize *dims, bool cplx) {
    return mxCreateNumericArray(ndim, dims, mxSINGLE_CLASS, cplx ? mxCOMPLEX : mxREAL);
}

// sizes of the last upload (for the outputs of 'run_*')
int g_n = 0, g_nz = 0, g_npos = 0;

void upload(const mxArray *S, const mxArray *cells) {
    const mxArray *rv = field(S, "RVol");
    if (mxGetNumberOfDimensions(rv) < 2) mexErrMsgTxt("RVol must be n x n x nz");
    const mwSize *d = mxGetDimensions(rv);
    const int n = (int)d[0];
    const int nz = mxGetNumberOfDimensions(rv) > 2 ? (int)d[2] : 1;
    const std::vector<float> rvol = to_single(rv);
    const std::vector<float> sx = to_single(field(S, "scan_xlist")), sy = to_single(field(S, "scan_ylist"));
    const std::vector<float> step = to_single(field(S, "step_size"));
    mset_upload_args a;
    std::memset(&a, 0, sizeof a);
    a.n = n;
    a.nz = nz;
    a.num_scan_pos = (int)scalar(S, "num_scan_pos");
    a.N_scan_x = (int)scalar(S, "N_scan_x");
    a.N_scan_y = (int)scalar(S, "N_scan_y");
    a.sigma = scalar(S, "sigma");
    a.potential_pixelsize = scalar(S, "potential_pixelsize");
    a.alpha = scalar(S, "alpha");  // read and unused, as in the reference
    a.E0 = scalar(S, "E0");
    for (int i = 0; i < 3 && i < (int)step.size(); ++i) a.step_size[i] = step[i];
    a.slice_binning = (int)scalar(S, "slice_binning");
    a.RVol = rvol.data();
    a.init_wave2D = complex_single(S, "init_wave2D");
    a.prop2D = complex_single(S, "prop2D");
    if ((int)sx.size() < a.num_scan_pos || (int)sy.size() < a.num_scan_pos)
        mexErrMsgTxt("scan_xlist / scan_ylist shorter than num_scan_pos");
    a.scan_xlist = sx.data();
    a.scan_ylist = sy.data();
    // cell k = position k; patterns of another class are converted (kept for the call)
    if ((int)mxGetNumberOfElements(cells) < a.num_scan_pos) mexErrMsgTxt("fewer measured patterns than positions");
    std::vector<const float *> table(a.num_scan_pos);
    std::vector<std::vector<float>> converted;
    converted.reserve(a.num_scan_pos);
    for (int k = 0; k < a.num_scan_pos; ++k) {
        const mxArray *c = mxGetCell(cells, (mwIndex)k);
        if (!c || mxGetNumberOfElements(c) != (size_t)n * n) mexErrMsgTxt("a measured pattern is not n x n");
        if (mxGetClassID(c) == mxSINGLE_CLASS) {
            table[k] = mxGetSingles(c);
        } else {
            converted.push_back(to_single(c));
            table[k] = converted.back().data();
        }
    }
    if (mset_mex_upload_cells(&a, table.data())) mexErrMsgTxt(mset_last_error());
    g_n = n;
    g_nz = nz;
    g_npos = a.num_scan_pos;
}

void run(int nlhs, mxArray *plhs[], int mode) {
    const mwSize rec_dims[3] = {(mwSize)g_n, (mwSize)g_n, (mwSize)g_nz};
    const mwSize probe_dims[2] = {(mwSize)g_n, (mwSize)g_n};
    const mwSize pos_dims[1] = {(mwSize)g_npos};
    const mwSize one[1] = {1};
    plhs[0] = single_array(3, rec_dims, false);
    plhs[1] = single_array(2, probe_dims, true);
    plhs[2] = single_array(1, pos_dims, false);
    plhs[3] = single_array(1, pos_dims, false);
    float *err = nullptr;
    if (nlhs == 5) {
        plhs[4] = single_array(1, one, false);
        err = mxGetSingles(plhs[4]);
    }
    if (mset_mex_run(mode, mxGetSingles(plhs[0]), reinterpret_cast<float *>(mxGetComplexSingles(plhs[1])),
                     mxGetSingles(plhs[2]), mxGetSingles(plhs[3]), err))
        mexErrMsgTxt(mset_last_error());
}

void error(mxArray *plhs[], int mode) {
    const mwSize one[1] = {1};
    plhs[0] = single_array(1, one, false);
    if (mset_mex_error(mode, mxGetSingles(plhs[0]))) mexErrMsgTxt(mset_last_error());
}

}  // namespace

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    if (nrhs < 1 || !mxIsChar(prhs[0])) mexErrMsgTxt("first argument: the mode string");
    char *m = mxArrayToString(prhs[0]);
    const std::string mode(m ? m : "");
    mxFree(m);
    if (mode == "upload") {
        if (nrhs < 3 || !mxIsStruct(prhs[1])) mexErrMsgTxt("upload needs STEM_data and the measured cell");
        upload(prhs[1], prhs[2]);
    } else if (mode == "run_mset") {
        run(nlhs, plhs, MSET_MODE_MSET);
    } else if (mode == "run_sset") {
        run(nlhs, plhs, MSET_MODE_SSET);
    } else if (mode == "error_mset") {
        error(plhs, MSET_MODE_MSET);
    } else if (mode == "error_sset") {
        error(plhs, MSET_MODE_SSET);
    } else {
        mexErrMsgTxt("The running mode is not correct (choose 'upload' or 'run_mset' or 'run_sset' or "
                     "'error_mset' or 'error_sset')");
    }
}
