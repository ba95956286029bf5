// Test infrastructure: a host entry point for the reference's vendored
// FastQSL adaptive field-line tracer (third_party/FastQSL/fastqslpy/cu/
// TraceBlineAdaptive.cu, driven by nfgs/_backend/util/fastqsl_plane.py:
// 203-383 through CuPy, which this image lacks).  The reference kernel is
// compiled unmodified from its own source file; this file only launches it
// with the grid that fastqsl_plane.py:196-200 uses (block_x threads per
// block, ceil(n / block_x) blocks), so that fixture scripts can run the
// reference tracer through ctypes on device buffers.  Nothing in the product
// links or calls this library.
#include "TraceBlineAdaptive.cu"

extern "C" int fq_ref_trace_all(float* bx, float* by, float* bz, int* bshape, float* cur_x, float* cur_y,
                                float* cur_z, double* twist, bool* cur_flag, float* inp_x, float* inp_y,
                                float* inp_z, float* normal, float* start_x, float* start_y, float* start_z,
                                int* flag_start, float* end_x, float* end_y, float* end_z, int* flag_end,
                                float* b_this_x, float* b_this_y, float* b_this_z, int* b_flag, float* b_start_x,
                                float* b_start_y, float* b_start_z, float* b_end_x, float* b_end_y, float* b_end_z,
                                float* step, unsigned long long* n_dev, double* line_len, float* tol,
                                long long n_points, int block_x, void* stream) {
    if (n_points <= 0 || block_x <= 0) return -1;
    const unsigned grid = (unsigned)((n_points + block_x - 1) / block_x);
    TraceAllBline<<<dim3(grid, 1, 1), dim3(block_x, 1, 1), 0, (cudaStream_t)stream>>>(
        bx, by, bz, bshape, cur_x, cur_y, cur_z, twist, cur_flag, inp_x, inp_y, inp_z, normal, start_x, start_y,
        start_z, flag_start, end_x, end_y, end_z, flag_end, b_this_x, b_this_y, b_this_z, b_flag, b_start_x,
        b_start_y, b_start_z, b_end_x, b_end_y, b_end_z, step, n_dev, line_len, tol);
    return (int)cudaGetLastError();
}
