// C-linkage entry points into the reference's own CPU implementation
// (src/few/cutils/interpolate.hh:27-38, AmpInterp2D.hh:6-8, gpuAAK.hh:6-10), so the oracle tests can call it
// through ctypes.  Built only by oracle/Makefile into oracle/_ref; test
// infrastructure, never part of the product path.
#include "AmpInterp2D.hh"
#include "interpolate.hh"

// gpuAAK.cu's get_waveform (gpuAAK.hh:6-10), compiled under the name aak_get_waveform
void aak_get_waveform(cmplx *waveform, double *interp_array, double M_phys, double S_phys, double mu, double qS,
                      double phiS, double qK, double phiK, double dist, int nmodes, bool mich, int init_len,
                      int out_len, double delta_t, double *h_t);

extern "C" {

void few_ref_aak_waveform(void *waveform, double *interp_array, double M_phys, double S_phys, double mu, double qS,
                          double phiS, double qK, double phiK, double dist, int nmodes, int mich, int init_len,
                          int out_len, double delta_t, double *h_t)
{
    aak_get_waveform((cmplx *)waveform, interp_array, M_phys, S_phys, mu, qS, phiS, qK, phiK, dist, nmodes,
                     mich != 0, init_len, out_len, delta_t, h_t);
}


void few_ref_interpolate_arrays(double *t_arr, double *interp_array, int ninterps, int length,
                                double *B, double *upper_diag, double *diag, double *lower_diag)
{
    interpolate_arrays(t_arr, interp_array, ninterps, length, B, upper_diag, diag, lower_diag);
}

void few_ref_interp2d(double *z, const double *tx, int nx, const double *ty, int ny, double *c, int kx, int ky,
                      const double *x, int mx, const double *y, int my, int num_indiv_c, int len_indiv_c)
{
    interp2D_wrap(z, tx, nx, ty, ny, c, kx, ky, x, mx, y, my, num_indiv_c, len_indiv_c);
}

void few_ref_get_waveform_fd(void *waveform, double *interp_array, double *phase_interp_t,
                             double *phase_interp_coeffs, int *m, int *k, int *n, int num_teuk_modes,
                             double delta_t, double *old_time_arr, int init_length, int data_length,
                             double *frequencies, int *seg_start_inds, int *seg_end_inds, int num_segments,
                             void *ylms, int zero_index, int include_minus_m, int separate_modes)
{
    get_waveform_generic_fd((cmplx *)waveform, interp_array, phase_interp_t, phase_interp_coeffs, m, k, n,
                            num_teuk_modes, delta_t, old_time_arr, init_length, data_length, frequencies,
                            seg_start_inds, seg_end_inds, num_segments, (cmplx *)ylms, zero_index,
                            include_minus_m != 0, separate_modes != 0);
}

void few_ref_get_waveform(void *d_waveform, double *interp_array, double *phase_interp_t,
                          double *phase_interp_coeffs, int *d_m, int *d_k, int *d_n, int init_len,
                          int out_len, int num_teuk_modes, void *d_Ylms, double delta_t, double *h_t,
                          int dev)
{
    get_waveform((cmplx *)d_waveform, interp_array, phase_interp_t, phase_interp_coeffs, d_m, d_k,
                 d_n, init_len, out_len, num_teuk_modes, (cmplx *)d_Ylms, delta_t, h_t, dev);
}

}
