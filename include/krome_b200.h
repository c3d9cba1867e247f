/* libkrome_b200_<net>.so -- the drop-in C ABI of the per-cell chemistry and
 * gas-temperature solve, computed on a B200 (sm_100a).
 *
 * One library per generated network (krome_x_b200/networks/net_<net>.h),
 * as the reference builds one libkrome per generated project. The entry
 * points below keep the reference's names, argument meanings, array
 * layouts and return flags; each cites the reference declaration it
 * replaces (runtime/interfaces/C/krome.h in the reference tree). The
 * krome_b200_* entry points are additions of this library.
 *
 * Layouts (as the reference): n[ncell][nspec] cell-major, species in the
 * network's code-point order; Tgas, dt [ncell]; par one row broadcast to
 * every cell (par_stride 0) or rows [ncell][npar] (par_stride npar).
 * Flags: 0 success; CVODE's -1 ... -27 for a failed integration (the cell
 * left untouched); -105 a REQUIRED parameter unset in some row (nothing
 * integrated); -110 the integration ended at Tgas <= 0; -104 a
 * configuration this library does not run (LAPACK linsol; sparse linsol on
 * the small networks, dense on the large) or no usable GPU; -111 the device
 * buffers could not be allocated; -1 bad arguments. There is no CPU
 * fallback. The conserve key (0 off, 1 the electrons restore the input net
 * charge, 2 the projection onto the input element totals and charge, 3 the
 * electrons neutralize the ions) applies to the cells that succeed, as the
 * reference's post-solve rule (solve_cell.hpp:1458-1500).
 */
#ifndef KROME_B200_H
#define KROME_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct krome_opts krome_opts;

/* ---- network description (reference krome.h:96-114) ---- */
/* krome.h:96 */
const char* krome_flag_message(int flag);
/* krome.h:99 */
const char* krome_version(void);
/* krome.h:101 */
const char* krome_network_name(void);
/* krome.h:102-104 */
int krome_nspec(void);
int krome_nrea(void);
int krome_npar(void);
/* krome.h:105-108 */
const char* krome_species_name(int i);
int krome_species_index(const char* name);
const char* krome_param_name(int i);
int krome_param_index(const char* name);
/* krome.h:111: one row of npar defaults; a REQUIRED parameter is NaN */
void krome_params_default(double* par);
/* krome.h:114 */
const char* krome_param_required_by(int i);

/* ---- options (reference krome.h:170-173, keys krome.cpp:198-260) ----
 * Keys as the reference: evolve_T, jac (0 auto, 1 analytic, 2 fd), linsol
 * (0 auto, 1 dense; 2 lapack and 3 sparse return -104 from a solve),
 * rtol, atol_n, atol_T, atol_u, max_steps, max_err_fails, max_conv_fails,
 * max_restarts, clip_negative, error_report, renormalize_x, conserve,
 * path, device_cache, device_memory, min_device, min_interleave. This
 * library's keys: layout (0 one warp per cell, 1 one lane per cell),
 * kernel (0 plain, 1 persistent work queue), lane_minb (2, 3, 4: the
 * lane kernel's register budget), queue_chunk, blocks_per_sm, fail_every
 * (fault injection: every k-th cell reports -1 untouched), lu32 (the Newton
 * matrix factored in FP32 with residuals, rhs, history and error test in
 * FP64; after a Newton failure the matrix is refactored in FP64 until the
 * next accepted step; lane layout only, else -104). Unknown key or bad
 * value: -1. */
krome_opts* krome_opts_new(void);
void krome_opts_free(krome_opts* h);
int krome_opts_set(krome_opts* h, const char* key, double value);
int krome_opts_get(const krome_opts* h, const char* key, double* value);
/* krome.h:175-185: per-species tolerances atol[NSPEC] / rtol[NSPEC] (a
 * negative entry: the scalar atol_n / rtol; NULL: the scalar for every
 * species); set rejects NaN and a zero atol with -1; get writes the
 * tolerance each species gets. Networks of up to 64 species (the large
 * networks' solve returns -104 with them set). */
int krome_opts_set_atol_species(krome_opts* h, const double* atol);
int krome_opts_set_rtol_species(krome_opts* h, const double* rtol);
int krome_opts_get_atol_species(const krome_opts* h, double* atol);
int krome_opts_get_rtol_species(const krome_opts* h, double* rtol);

/* the optional per-cell arrays of a call (reference krome.h:258-294):
 * Phi[ncell][nbins] the photon flux per bin, read with photon bins on the
 * handle (krome_opts_set_photo); Td and adust (binned dust, not built in
 * this library) are not read. NULL, or unused members NULL. */
typedef struct {
  double* Phi;
  double* Td;
  double* adust;
} krome_cells;

/* ---- the solve (reference krome.h:291-294, krome.cpp:396-438) ----
 * Host arrays, updated in place; extra (krome_cells) may be NULL;
 * flags[ncell] may be NULL. Returns 0 or the lowest-index failing cell's
 * flag. */
int krome_solve_cells(int ncell, double* n, double* Tgas, const double* dt,
                      const double* par, int par_stride, const krome_cells* extra,
                      int* flags, const krome_opts* h);

/* krome_solve_cells with mass fractions (reference krome.h:302-306):
 * x[ncell][nspec] and the gas density rho[ncell] [g cm^-3]; n = rho x / m
 * on the way in (0 for a species without mass), x = m n / rho on the way
 * out for the cells that succeed (rescaled to the input sum of the
 * fractions with the renormalize_x key); a failed cell keeps its input x.
 * Host arrays; flags may be NULL. */
int krome_solve_cells_x(int ncell, double* x, const double* rho,
                        double* Tgas, const double* dt, const double* par,
                        int par_stride, const krome_cells* extra, int* flags,
                        const krome_opts* h);

/* ---- device-resident data (reference krome.h:308-349) ----
 * krome_solve_cells and _x on arrays in device memory, in one of two
 * layouts: species-major n[i * ld + c] (ld >= ncell; 0: ncell, a Fortran
 * n(ld, nspec)) or cell-major n[c * nspec + i]. Tgas, dt (and rho) [ncell]
 * on the device; par device rows (par_stride 0 or npar) or NULL for the
 * defaults; extra->Phi the cells' photon field (device rows, with photon
 * bins on the handle); flags[ncell] on the device, may be NULL;
 * summary (host, may be NULL) counts the cells: solved on the device,
 * recovered on the host (always 0: there is no CPU fallback), failed. The
 * lane-per-cell kernel (the default) reads and writes the caller's layout
 * and converts mass fractions itself; the other kernels stage through
 * cell-major copies. The device is synchronized before and after the
 * call. Returns 0, the lowest failing cell's flag, -105 (a required
 * parameter unset in some row: nothing integrated), -104 (unsupported
 * configuration or a CUDA error), -111 (no device memory for the staging
 * buffer) or -1 (bad arguments). */
#define KROME_LAYOUT_SPECIES_MAJOR 0
#define KROME_LAYOUT_CELL_MAJOR 1
typedef struct {
  long device; /* cells solved on the device */
  long host;   /* failed on the device, solved on the host (0 here) */
  long failed; /* failed */
} krome_device_summary;
/* krome.h:339-344 */
int krome_solve_cells_device(int ncell, double* n, int layout, long ld,
                             double* Tgas, const double* dt,
                             const double* par, int par_stride,
                             const krome_cells* extra, int* flags,
                             krome_device_summary* summary,
                             const krome_opts* h);
/* krome.h:345-350 */
int krome_solve_cells_x_device(int ncell, double* x, const double* rho,
                               int layout, long ld, double* Tgas,
                               const double* dt, const double* par,
                               int par_stride, const krome_cells* extra,
                               int* flags, krome_device_summary* summary,
                               const krome_opts* h);

/* krome.h:351-360: krome_conserve_cells and _x (below) on device arrays in
 * either layout above; ref [rows][nelem], par and flags on the device too.
 * One thread per cell; the device is synchronized before the call. Returns
 * the lowest failing cell's flag (negative), 0, -104 (a CUDA error) or -1
 * (bad arguments). */
int krome_conserve_cells_device(int ncell, double* n, int layout, long ld,
                                const double* ref, int ref_stride,
                                const double* par, int par_stride,
                                int* flags);
int krome_conserve_cells_x_device(int ncell, double* x, int layout, long ld,
                                  const double* ref, int ref_stride,
                                  const double* par, int par_stride,
                                  int* flags);

/* krome_get_rates (reference krome.h:387-389): k[ncell][nrea] at each
 * cell's rate temperature clamp(Tgas, Tcmb, 1e9), the photo rates of
 * Phi[ncell][nbins] with photon bins on h (-103 without a field) */
int krome_get_rates(int ncell, const double* n, const double* Tgas,
                    const double* par, int par_stride, const double* Phi,
                    const krome_opts* h, double* k);

/* krome_has_device (reference krome.h:193): 1 when a CUDA device is
 * visible */
int krome_has_device(void);

/* ---- host utilities (reference krome.h:473-501, 539, 645-652) ---- */
/* krome.h:476-477: tot[ncell][nelem] element totals [atoms cm^-3], or per
 * gram [atoms g^-1] from mass fractions */
int krome_get_element_totals(int ncell, const double* n, double* tot);
int krome_get_element_totals_x(int ncell, const double* x, double* tot);
/* krome.h:478-497: consistent advection -- each cell moved to its reference
 * element totals ref (ref_stride 0 one row, nelem a row per cell) and to
 * zero net charge; flags 0, -112 (unreachable: corrected as far as
 * possible) or the warning 2 (a species changed by more than 50 %); par
 * may be NULL (no freeze directives in these networks) */
int krome_conserve_cells(int ncell, double* n, const double* ref,
                         int ref_stride, const double* par, int par_stride,
                         int* flags);
int krome_conserve_cells_x(int ncell, double* x, const double* ref,
                           int ref_stride, const double* par, int par_stride,
                           int* flags);
/* krome.h:501, 539: x = m n / rho and back, rho[ncell] [g cm^-3] */
int krome_n2x(int ncell, const double* n, const double* rho, double* x);
int krome_x2n(int ncell, const double* x, const double* rho, double* n);
/* krome.h:646-652: species mass [g] (NaN out of range), charge, elements */
double krome_species_mass(int i);
int krome_species_charge(int i);
int krome_nelem(void);
const char* krome_element_name(int e);
int krome_species_natoms(int i, int e);
/* krome.h:194-201: the device backend's set-up; this library needs none:
 * 0 with a usable device (-104 without); _id makes the device current */
int krome_device_initialize(void);
int krome_device_initialize_id(int device_id);
int krome_device_finalize(void);

/* ---- the rest of the reference's interface: metadata, queries and the
 * photon-field helpers (evaluated on the host; rates at clamp(Tgas, Tcmb,
 * 1e9), thermal terms at clamp(Tgas, 2.73, 1e9), as the solve) ---- */
/* krome.h:651 */
const char* krome_reaction_name(int r);
/* krome.h:405-418: the active thermal terms (names in the reference's
 * order), their values, the adiabatic index, the per-reaction energy
 * release (none in these networks: 0) */
int krome_nheat(void);
int krome_ncool(void);
const char* krome_heating_name(int i);
const char* krome_cooling_name(int i);
int krome_get_thermal(int ncell, const double* n, const double* Tgas,
                      const double* par, int par_stride, const double* Phi,
                      const krome_opts* h, double* heat, double* cool,
                      double* heats, double* cools, double* dTdt);
int krome_get_qeff(int ncell, const double* n, const double* Tgas,
                   const double* par, int par_stride, double* q);
int krome_get_gamma(int ncell, const double* n, const double* Tgas,
                    const double* par, int par_stride, double* gamma);
/* krome.h:390, 397: reaction fluxes k prod(n); the dust temperature the
 * rates see (the Tdust parameter; -1 for a network without one) */
int krome_get_fluxes(int ncell, const double* n, const double* Tgas,
                     const double* par, int par_stride, const double* Phi,
                     const krome_opts* h, double* fl);
int krome_get_Tdust(int ncell, const double* n, const double* Tgas,
                    const double* par, int par_stride, const double* Phi,
                    const krome_opts* h, double* Td);
/* krome.h:424-438: per-cell quantities of the densities */
int krome_get_mu(int ncell, const double* n, double* out);
int krome_get_rho(int ncell, const double* n, double* out);
int krome_get_ntot(int ncell, const double* n, double* out);
int krome_get_Hnuclei(int ncell, const double* n, double* out);
int krome_get_charge(int ncell, const double* n, double* out);
int krome_get_electrons(int ncell, const double* n, double* out);
int krome_get_free_fall_time(int ncell, const double* n, double* out);
int krome_get_jeans_length(int ncell, const double* n, const double* Tgas,
                           double* out);
int krome_get_free_fall_time_rho(int ncell, const double* rho, double* out);
int krome_num2col(int ncell, const double* num, const double* n,
                  const double* Tgas, const double* par, int par_stride,
                  double* out);
/* krome.h:521: the neutral atomic metals at metallicity Z */
int krome_scale_Z(int ncell, double* n, double Z);
/* krome.h:449-458: line coolants of coolant files (none here: 0 coolants,
 * -1 for any index) */
int krome_ncoolant(void);
const char* krome_coolant_name(int i);
int krome_coolant_species(int i);
int krome_coolant_nlev(int i);
int krome_coolant_levels(int i, double* E, double* g);
int krome_get_coolant_cooling(int ncell, const double* n, const double* Tgas,
                              const double* par, int par_stride,
                              const double* Phi, const krome_opts* h,
                              double* cool);
int krome_get_coolant_populations(int ncell, const double* n,
                                  const double* Tgas, const double* par,
                                  int par_stride, const double* Phi,
                                  const krome_opts* h, int i, double* pop);
/* krome.h:548-595: photon-field helpers (bins, J <-> Phi, spectra integrated
 * over the bins, dust opacity per bin, the G0 / Av fit); the Haardt &
 * Madau 2012 background and the Draine dust opacity need tables this
 * library does not carry: -104 */
int krome_bins_lin(int nbins, double lower, double upper, double* Elo,
                   double* Ehi);
int krome_bins_log(int nbins, double lower, double upper, double* Elo,
                   double* Ehi);
int krome_J_to_phi(int nbins, const double* Elo, const double* Ehi,
                   const double* J, double* phi);
int krome_phi_to_J(int nbins, const double* Elo, const double* Ehi,
                   const double* phi, double* J);
int krome_spectrum_blackbody(int nbins, const double* Elo, const double* Ehi,
                             double Tbb, double* phi);
int krome_blackbody_range(double Tbb, double* lower, double* upper);
int krome_spectrum_draine(int nbins, const double* Elo, const double* Ehi,
                          double* phi);
int krome_spectrum_j21(int nbins, const double* Elo, const double* Ehi,
                       double J21, double alpha, double* phi);
int krome_spectrum_hm2012(int nbins, const double* Elo, const double* Ehi,
                          double z, double* phi);
int krome_spectrum_table(int nbins, const double* Elo, const double* Ehi,
                         int nE, const double* E, const double* J,
                         int loglog, double* phi);
int krome_dust_kappa_bins(int nE, const double* E, const double* kappa,
                          int nbins, const double* Elo, const double* Ehi,
                          double* kbin);
int krome_dust_kappa_draine(int nbins, const double* Elo, const double* Ehi,
                            double* kbin);
int krome_find_G0_Av(int nbins, const double* Elo, const double* Ehi,
                     const double* phi, const double* kbin, double d2g,
                     double xH, double* G0, double* Av);
/* krome.h:602-640: the photo reactions, J_LW rates (none here), photon
 * bins on the handle and the field queries */
int krome_nphoto(void);
int krome_photo_reaction(int r);
int krome_photo_reactant(int r);
double krome_photo_pdiss(int r);
double krome_photo_xsec(int r, double E);
int krome_nlw(void);
int krome_lw_reaction(int q);
int krome_lw_reactant(int q);
double krome_lw_pdiss(int q);
/* krome.h:206-228 */
int krome_opts_set_photo(krome_opts* h, int nbins, const double* Elo,
                         const double* Ehi);
int krome_opts_nbins(const krome_opts* h);
int krome_opts_set_photo_broadening(krome_opts* h, double Tgas, double vturb);
int krome_opts_set_photo_alpha(krome_opts* h, double alpha);
int krome_opts_set_photo_dust_opacity(krome_opts* h, const double* kappa);
int krome_opts_lw_weights(const krome_opts* h, double* w);
int krome_opts_photo_sigma(const krome_opts* h, double* sigma);
int krome_get_photo_heating(int ncell, const double* n, const double* Tgas,
                            const double* par, int par_stride,
                            const double* Phi, const krome_opts* h,
                            double* heat);
int krome_get_ratio_flux_draine(int ncell, const double* Phi,
                                const krome_opts* h, double* ratio);
int krome_get_habing(int ncell, const double* Phi, const krome_opts* h,
                     double* G);
int krome_get_opacity(int ncell, const double* n, const double* Tgas,
                      const double* par, int par_stride, const krome_opts* h,
                      const double* d2g, const double* kdust, double* tau);
int krome_get_absorption(int ncell, const double* n, const double* Tgas,
                         const double* par, int par_stride,
                         const krome_opts* h, const double* kdust,
                         double* kabs);
/* krome.h:236-256: binned dust is not built in this library: set returns
 * -104, ndust 0, the rest -1 (as without bins) */
int krome_opts_set_dustbins(krome_opts* h, int nd, int use_Si, int use_C,
                            double alow, double aup, double phi);
int krome_opts_ndust(const krome_opts* h);
int krome_opts_set_dust_Td(krome_opts* h, const double* Td);
int krome_opts_get_dust_Td(const krome_opts* h, double* Td);
int krome_opts_set_dust_a(krome_opts* h, const double* a);
int krome_opts_get_dust_a(const krome_opts* h, double* a);
int krome_opts_get_dust_counts(const krome_opts* h, double rho_gas,
                               double d2g, double* nd);
int krome_opts_get_dust_types(const krome_opts* h, int* isC);
/* krome.h:364: the error-report file name (kept; no report is written) */
int krome_opts_set_error_file(krome_opts* h, const char* path);
/* krome.h:373: integrate every cell to steady state (eq_* keys) */
int krome_equilibrium_cells(int ncell, double* n, double* Tgas,
                            const double* par, int par_stride,
                            const krome_cells* extra, int* flags,
                            const krome_opts* h);

/* ---- additions of this library ---- */

/* the number of per-cell counters, and the equations of a cell */
int krome_b200_nstat(void);
int krome_b200_neq(int evolve_T);

/* krome_solve_cells with per-cell counters: stats[ncell][nstat] (nst, nfe,
 * nfeDQ, nje, nsetups, nni, nnf, netf, restarts, nlu64 = the FP64 refactors
 * of the lu32 form; may be NULL). The
 * batched entry point the Python binding's solve / solve_batch use. */
int krome_b200_solve_batch(int ncell, double* n, double* Tgas,
                           const double* dt, const double* par,
                           int par_stride, int* flags, long* stats,
                           const krome_opts* h);

/* device-resident solve (the role of the reference's
 * krome_solve_cells_device, krome.h:339-344, cell-major layout): every
 * pointer is device memory, n and Tgas updated in place, flags[ncell]
 * (required), stats optional, cursor one unsigned (the persistent
 * kernel's work queue; reset by the call). Asynchronous on `stream` (a
 * cudaStream_t, NULL the legacy stream); no host synchronization, so it
 * can be captured in a CUDA graph. The required-parameter rule is checked
 * per cell on the device (-105 in that cell's flag). Returns 0 after a
 * successful launch, -1 bad arguments, -104 launch failure. */
int krome_b200_solve_device(int ncell, double* n, double* Tgas,
                            const double* dt, const double* par,
                            int par_stride, int* flags, long* stats,
                            unsigned* cursor, const krome_opts* h,
                            void* stream);

/* one step of the reference's collapse driver on device arrays
 * (examples/tests/collapse/test.cpp:47-63): tff = the free-fall time of
 * each cell's current densities written into parameter tff_index, every
 * density x factor, dt = dtfrac tff, then krome_b200_solve_device.
 * par must be per-cell rows (par_stride npar). Asynchronous on stream. */
int krome_b200_hydro_step(int ncell, double* n, double* Tgas, double* dt,
                          double* par, int par_stride, int tff_index,
                          double factor, double dtfrac, int* flags,
                          long* stats, unsigned* cursor, const krome_opts* h,
                          void* stream);

/* krome_b200_hydro_step captured once as a CUDA graph on `stream` (a
 * non-default stream) and replayed with krome_b200_graph_launch; the arrays
 * stay bound to the graph. new returns NULL on failure. */
void* krome_b200_graph_new(int ncell, double* n, double* Tgas, double* dt,
                           double* par, int par_stride, int tff_index,
                           double factor, double dtfrac, int* flags,
                           long* stats, unsigned* cursor, const krome_opts* h,
                           void* stream);
int krome_b200_graph_launch(void* graph, void* stream);
void krome_b200_graph_free(void* graph);

/* ---- the discrete adjoint (no counterpart in the reference, whose only
 * rate scaling is a global factor) ----
 * The solve of krome_b200_solve_batch with every rate coefficient k_r of
 * cell c multiplied by exp(lnm[c][r]), and the gradient of
 * sum(gn * n_out) + sum(gT * Tgas_out) with respect to the initial n
 * (dn0[ncell][nspec]), Tgas (dT0[ncell], evolve_T) and lnm
 * (dm[ncell][nrea], per cell). The gradient is that of the discrete
 * solution: the forward solve's step sizes, orders and Newton decisions are
 * held fixed, each accepted step's corrector is differentiated at its root
 * with dF/dy re-evaluated at the accepted state. lnm: one row of nrea
 * (lnm_stride 0) or rows (nrea), NULL for none. tape_cap: doubles of tape
 * per cell (0: 32768); a cell whose tape outgrows it returns -120 untouched.
 * Failed cells get zero gradients. Host arrays; the device buffers (the
 * tapes: ncell * tape_cap * 8 bytes) are allocated per call. Returns 0 or
 * the lowest-index failing cell's flag. */
int krome_b200_adjoint(int ncell, double* n, double* Tgas, const double* dt,
                       const double* par, int par_stride, const double* lnm,
                       int lnm_stride, const double* gn, const double* gT,
                       int* flags, double* dn0, double* dT0, double* dm,
                       long tape_cap, const krome_opts* h);

/* the adjoint's two halves on device arrays, asynchronous on `stream`:
 * the recording forward solve (mult = exp(lnm), rows [ncell][nrea] with
 * mult_stride nrea or one row with 0, NULL for none; tape[ncell][tape_cap];
 * tape_len[ncell] and yfin[ncell][neq] written for the reverse sweep;
 * n, Tgas updated in place as by krome_b200_solve_device; tape NULL: a
 * counting solve, tape_len[c] the doubles cell c's tape needs) ... */
int krome_b200_adjoint_record_device(int ncell, double* n, double* Tgas,
                                     const double* dt, const double* par,
                                     int par_stride, const double* mult,
                                     int mult_stride, int* flags, long* stats,
                                     unsigned* cursor, double* tape,
                                     long tape_cap, long* tape_len,
                                     double* yfin, const krome_opts* h,
                                     void* stream);
/* ... and the reverse sweep over those tapes (T0: the initial Tgas;
 * cursor: one unsigned, the sweep's work queue, reset by the call) */
int krome_b200_adjoint_device(int ncell, const double* T0, const double* par,
                              int par_stride, const double* mult,
                              int mult_stride, const double* gn,
                              const double* gT, const int* flags,
                              const double* tape, long tape_cap,
                              const long* tape_len, const double* yfin,
                              double* dn0, double* dT0, double* dm,
                              unsigned* cursor, const krome_opts* h,
                              void* stream);

/* krome_solve_cells for callers that cannot let the library allocate device
 * memory -- a code that gives the whole GPU to its own memory pool, or a
 * time step that must not pay cudaMalloc's device-wide synchronization.
 * No counterpart in the reference (its device path allocates per call).
 * The arguments of krome_solve_cells without `extra` (no photon or dust
 * rows); same layouts, flags and failed-cell rule (flags may be NULL). The
 * call's device copies go through one array compiled into the library,
 * 16 MiB of device memory per GPU held until the process exits, instead of
 * an allocation: it fits about 16 MiB / (8 (nspec + 2 + npar) + 4)
 * bytes-per-cell cells (per-cell parameter rows), and a larger call returns
 * -111 (FLAG_DEVICE_MEMORY) with nothing touched. Call it once with
 * ncell == 0 on each device (that device current) before the caller's pool
 * takes the GPU and before any stream capture: it looks up the array's
 * device address, which loads the library's device code, and launches the
 * kernel the options select once with no cells, so that the driver
 * reserves the kernel's per-thread local memory then; it returns 0, or the
 * flag the options would give (-104). All calls share the array: the entry
 * point serialises its own calls, and calls that overlapped on the GPU
 * would race. Results come back through host staging: a failed copy leaves
 * the caller's arrays untouched (-104). The large networks (the sparse
 * path, whose workspace this cannot provide) return -104 in every flag. */
int krome_b200_solve_cells_noalloc(int ncell, double* n, double* Tgas,
                                   const double* dt, const double* par,
                                   int par_stride, int* flags,
                                   const krome_opts* h);

/* the network rhs evaluated alone, one thread per cell, reps times per
 * cell, at full SIMT width (host arrays of the evolve_T state): rhs
 * evaluations per second -- the rhs-throughput bound of the solve */
int krome_b200_rhs_throughput(int ncell, const double* n, const double* Tgas,
                              const double* par, int par_stride, int reps,
                              double* rhs_per_s);

/* the FP64 pipe's peak of this GPU, measured with register-resident DFMA
 * chains over the whole device [TFLOP/s] (the roofline's denominator) */
int krome_b200_fp64_peak(double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* KROME_B200_H */
