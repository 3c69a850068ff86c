// mex_shim.cpp -- minimal host implementation of the MEX API subset declared
// in mex.h, plus a C entry layer that builds the mxArrays the reference's
// mexFunction expects (src/CUDA/mex_main.cu:19-39) and copies its outputs back.
//
// TEST INFRASTRUCTURE ONLY: links the reference's unchanged CUDA sources into
// oracle/_ref/libmset_ref.so, used by the GPU parity tests and as a timed
// baseline.  Nothing under mset_b200/ loads it.
#include "mex.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

struct mxArray_tag {
    mxClassID cls = mxUNKNOWN_CLASS;
    bool cplx = false;
    std::vector<mwSize> dims;
    std::vector<unsigned char> data;          // numeric payload (interleaved if complex)
    std::vector<std::string> names;           // struct field names (1x1 struct)
    std::vector<mxArray *> fields;            // struct field values
    std::vector<mxArray *> cells;             // cell elements
    std::string str;                          // char arrays
};

namespace {

struct MexError : std::runtime_error {
    explicit MexError(const char *m) : std::runtime_error(m) {}
};

std::string g_last_error;
std::vector<std::unique_ptr<mxArray>> g_pool;     // arrays alive for the session
std::vector<std::unique_ptr<mxArray>> g_outputs;  // arrays created by mexFunction

size_t elem_size(mxClassID c) {
    switch (c) {
    case mxDOUBLE_CLASS: return 8;
    case mxSINGLE_CLASS: return 4;
    case mxINT8_CLASS: case mxUINT8_CLASS: case mxLOGICAL_CLASS: return 1;
    case mxINT16_CLASS: case mxUINT16_CLASS: return 2;
    case mxINT32_CLASS: case mxUINT32_CLASS: return 4;
    case mxINT64_CLASS: case mxUINT64_CLASS: return 8;
    default: return 0;
    }
}

size_t numel(const mxArray *a) {
    size_t n = 1;
    for (auto d : a->dims) n *= d;
    return n;
}

mxArray *make(std::vector<std::unique_ptr<mxArray>> &pool) {
    pool.emplace_back(new mxArray());
    return pool.back().get();
}

mxArray *make_single(std::vector<std::unique_ptr<mxArray>> &pool, std::vector<mwSize> dims,
                     const float *src, bool cplx) {
    mxArray *a = make(pool);
    a->cls = mxSINGLE_CLASS;
    a->cplx = cplx;
    a->dims = std::move(dims);
    size_t bytes = numel(a) * 4 * (cplx ? 2 : 1);
    a->data.resize(bytes);
    if (src) std::memcpy(a->data.data(), src, bytes);
    return a;
}

mxArray *make_scalar(std::vector<std::unique_ptr<mxArray>> &pool, float v) {
    return make_single(pool, {1, 1}, &v, false);
}

mxArray *make_string(std::vector<std::unique_ptr<mxArray>> &pool, const char *s) {
    mxArray *a = make(pool);
    a->cls = mxCHAR_CLASS;
    a->str = s;
    a->dims = {1, std::strlen(s)};
    return a;
}

// session inputs (the reference borrows the measured cell across calls,
// mex_main.cu:87)
mxArray *g_struct = nullptr;
mxArray *g_cells = nullptr;
int g_npos = 0;

int call(const char *mode, int nlhs, mxArray **plhs) {
    const mxArray *prhs[3];
    prhs[0] = make_string(g_pool, mode);
    prhs[1] = g_struct;
    prhs[2] = g_cells;
    try {
        mexFunction(nlhs, plhs, 3, prhs);
    } catch (const MexError &e) {
        g_last_error = e.what();
        return -1;
    }
    cudaError_t ce = cudaDeviceSynchronize();
    if (ce != cudaSuccess) {
        g_last_error = cudaGetErrorString(ce);
        return -2;
    }
    return 0;
}

}  // namespace

extern "C" {

void mexErrMsgTxt(const char *msg) { throw MexError(msg); }

mxArray *mxGetCell(const mxArray *pm, mwIndex index) {
    if (index >= pm->cells.size()) return nullptr;
    return pm->cells[index];
}
float *mxGetSingles(const mxArray *pm) { return (float *)pm->data.data(); }
mxComplexSingle *mxGetComplexSingles(const mxArray *pm) { return (mxComplexSingle *)pm->data.data(); }
double *mxGetDoubles(const mxArray *pm) { return (double *)pm->data.data(); }
uint8_t *mxGetUint8s(const mxArray *pm) { return (uint8_t *)pm->data.data(); }
int32_t *mxGetInt32s(const mxArray *pm) { return (int32_t *)pm->data.data(); }
mxLogical *mxGetLogicals(const mxArray *pm) { return (mxLogical *)pm->data.data(); }
void *mxGetData(const mxArray *pm) { return (void *)pm->data.data(); }

mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid, mxComplexity flag) {
    mxArray *a = make(g_outputs);
    a->cls = classid;
    a->cplx = flag == mxCOMPLEX;
    a->dims.assign(dims, dims + ndim);
    a->data.assign(numel(a) * elem_size(classid) * (a->cplx ? 2 : 1), 0);
    return a;
}
mxClassID mxGetClassID(const mxArray *pm) { return pm->cls; }
size_t mxGetNumberOfElements(const mxArray *pm) {
    if (pm->cls == mxCELL_CLASS) return pm->cells.size();
    return numel(pm);
}
mwSize mxGetNumberOfDimensions(const mxArray *pm) { return pm->dims.size(); }
const mwSize *mxGetDimensions(const mxArray *pm) { return pm->dims.data(); }
int mxGetNumberOfFields(const mxArray *pm) { return (int)pm->names.size(); }
const char *mxGetFieldNameByNumber(const mxArray *pm, int n) { return pm->names[n].c_str(); }
mxArray *mxGetFieldByNumber(const mxArray *pm, mwIndex, int n) { return pm->fields[n]; }
bool mxIsStruct(const mxArray *pm) { return pm->cls == mxSTRUCT_CLASS; }
bool mxIsChar(const mxArray *pm) { return pm->cls == mxCHAR_CLASS; }
char *mxArrayToString(const mxArray *pm) {
    // leaked per call unless the caller mxFree's it, as in MATLAB
    char *s = (char *)std::malloc(pm->str.size() + 1);
    std::memcpy(s, pm->str.c_str(), pm->str.size() + 1);
    return s;
}
void mxFree(void *ptr) { std::free(ptr); }

// ---------------------------------------------------------------------------
// C driver.  Array layouts are the MEX ones: C order [nz][n][n] for RVol
// (MATLAB size n x n x nz), [n][n] interleaved complex for the probe and the
// centred propagator, [npos][n][n] for the measured patterns (cell element k
// = position k, column-major cell of size nsx x nsy).
// ---------------------------------------------------------------------------
const char *ref_last_error(void) { return g_last_error.c_str(); }

int ref_upload(int n, int nz, const float *rvol, const float *probe, const float *prop,
               float sigma, float dz, int nsx, int nsy, int npos, const float *scan_x,
               const float *scan_y, const float *step3, int binning, const float *measured) {
    g_pool.clear();
    g_outputs.clear();
    g_struct = make(g_pool);
    g_struct->cls = mxSTRUCT_CLASS;
    g_struct->dims = {1, 1};
    auto add = [&](const char *name, mxArray *v) {
        g_struct->names.push_back(name);
        g_struct->fields.push_back(v);
    };
    mwSize un = (mwSize)n, unz = (mwSize)nz;
    add("RVol", make_single(g_pool, {un, un, unz}, rvol, false));
    add("init_wave2D", make_single(g_pool, {un, un}, probe, true));
    add("prop2D", make_single(g_pool, {un, un}, prop, true));
    add("alpha", make_scalar(g_pool, 0.f));
    add("sigma", make_scalar(g_pool, sigma));
    add("E0", make_scalar(g_pool, 300.f));
    add("potential_pixelsize", make_scalar(g_pool, dz));
    add("N_scan_x", make_scalar(g_pool, (float)nsx));
    add("N_scan_y", make_scalar(g_pool, (float)nsy));
    add("scan_xlist", make_single(g_pool, {(mwSize)npos, 1}, scan_x, false));
    add("scan_ylist", make_single(g_pool, {(mwSize)npos, 1}, scan_y, false));
    add("num_scan_pos", make_scalar(g_pool, (float)npos));
    add("step_size", make_single(g_pool, {1, 3}, step3, false));
    add("slice_binning", make_scalar(g_pool, (float)binning));
    g_cells = make(g_pool);
    g_cells->cls = mxCELL_CLASS;
    g_cells->dims = {(mwSize)nsx, (mwSize)nsy};
    for (int p = 0; p < npos; ++p)
        g_cells->cells.push_back(make_single(g_pool, {un, un}, measured + (size_t)p * n * n, false));
    g_npos = npos;
    return call("upload", 0, nullptr);
}

int ref_run(int mode, float *rvol_out, float *probe_out, float *scan_x_out, float *scan_y_out,
            float *err_out) {
    mxArray *plhs[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int nlhs = err_out ? 5 : 4;
    g_outputs.clear();
    int rc = call(mode == 2 ? "run_sset" : "run_mset", nlhs, plhs);
    if (rc) return rc;
    std::memcpy(rvol_out, plhs[0]->data.data(), plhs[0]->data.size());
    std::memcpy(probe_out, plhs[1]->data.data(), plhs[1]->data.size());
    std::memcpy(scan_x_out, plhs[2]->data.data(), plhs[2]->data.size());
    std::memcpy(scan_y_out, plhs[3]->data.data(), plhs[3]->data.size());
    if (err_out) std::memcpy(err_out, plhs[4]->data.data(), 4);
    return 0;
}

// any mode string with no outputs (the gateways' answer to an unknown mode)
int ref_mode(const char *mode) {
    g_outputs.clear();
    return call(mode, 0, nullptr);
}

int ref_error(int mode, float *err_out) {
    mxArray *plhs[1] = {nullptr};
    g_outputs.clear();
    int rc = call(mode == 2 ? "error_sset" : "error_mset", 1, plhs);
    if (rc) return rc;
    std::memcpy(err_out, plhs[0]->data.data(), 4);
    return 0;
}

}  // extern "C"
