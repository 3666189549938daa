/*
 * Diagnostic entry points of libpytme_b200.so for the test suite: single kernels of
 * the fused scan run on caller data. They are exported (the tests reach them through
 * ctypes) but are not part of the public interface in include/pytme_b200.h and have
 * no counterpart in the reference.
 */
#ifndef PYTME_B200_DIAGNOSTICS_H
#define PYTME_B200_DIAGNOSTICS_H

#ifdef __cplusplus
extern "C" {
#endif

/* Diagnostic: the tensor-core x pass alone (complex64 G [nb][t0][n1][h2] and C
 * [n0][n1][h2] in, H [nb][n0][n1][h2] complex64 or half2 out):
 * H[b][x'] = sum_{x<t0} scale * C[(x'-x) mod n0] * G[b][x] per column. Synchronises. */
int tm_xcorr_tc_test(const void* G, const void* C, int nb, int t0, int n0, int n1, int h2,
                     float scale, void* H, int half, void* stream);

/* Diagnostic: `lines` complex FFTs of length n (dir -1 forward, +1 unnormalised
 * inverse) with the shared-memory line-FFT routine of the fused scan.
 * Synchronises. */
int tm_line_fft_test(const void* x, void* y, int n, int lines, int dir, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PYTME_B200_DIAGNOSTICS_H */
