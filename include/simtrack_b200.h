/*
 * simtrack_b200 C ABI.
 *
 * The drop-in boundary for SimTrack's tracking path: plain C types, pointers
 * and sizes only.  Every entry point returns a status code (STB_OK or a
 * negative STB_E* value) and never terminates the process; the message of the
 * last failure on the calling thread is available from stb_last_error().
 * Each declaration names the reference interface it replaces
 * (simtrack.h / simtrack.cpp, file:line).
 *
 * Threading: the element and line objects are not synchronised; a table may
 * be used by one host thread at a time.  Device-pointer entry points take an
 * explicit cudaStream_t passed as void*.
 */
#ifndef SIMTRACK_B200_H
#define SIMTRACK_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STB_OK 0
#define STB_EINVAL (-1)
#define STB_ENOMEM (-2)
#define STB_ECUDA (-3)
#define STB_ETIMEOUT (-4)
#define STB_EABORTED (-5)
#define STB_EUNSUPPORTED (-6)

typedef struct stb_element stb_element; /* Element*  (simtrack.h:373-396) */
typedef struct stb_line stb_line;       /* Line      (simtrack.h:1067-1100) */
typedef struct stb_table stb_table;     /* flattened device element table (no reference counterpart) */
typedef struct stb_scan stb_scan;       /* batched dynamic-aperture scan (replaces the Track_DA* loops) */
typedef struct stb_mlp stb_mlp;         /* loss-prediction surrogate network (no reference counterpart) */

/* Message of the last failed call on this thread ("" if none). */
const char *stb_last_error(void);
/* Library version as major*10000 + minor*100 + patch. */
int stb_version(void);

/* ---- reference particle: GlobalVariables GP (simtrack.h:28-68) ---- */
/* Set_RefPartEnergy(gamma, E0, Q, A)  simtrack.cpp:87-108 */
int stb_set_ref_energy(double gamma, double E0, double Q, double A);
/* Set_Spin_G(g)  simtrack.cpp:110-115 */
int stb_set_spin_g(double g);
/* GP.H_expand, GP.quad_fringe  simtrack.h:62-66 (GP.radiate: stb_set_radiation) */
int stb_set_flags(int h_expand, int quad_fringe);

/* GP.radiate (simtrack.h:57): synchrotron radiation in the sector bends
 * (SBEND_Pass's radiating branch, simtrack.cpp:4740-4748: radiate1 with
 * quantum excitation after each of the Nint slices), in GMULT/SBENDMULT
 * (5312-5338, 5437-5463: radiate after each slice) and in GSBEND (4866-4873:
 * radiate2), for tables created after the call.  The reference draws the quantum-excitation deviates from GSL's
 * sequential stream (gsl_ran_gaussian on gsl_r2, seeded 1324 in
 * Init_GSL_Seeds, 317-329); here the k-th deviate of particle i (its index in
 * the arrays of the Track call, k counting its radiating slices from turn 0)
 * is a function of (seed, i, k): Philox4x32-10 and Box-Muller, the same on
 * every launch shape.  Radiating tables are tracked by the stb_track_* and
 * stb_track_spin_* entry points (spin tables: radiate after each slice's spin
 * rotation of SBEND and SBENDMULT, 7519-7529, 7887-7918), not by the scan,
 * Track_Radial or static ones.  GSBEND radiates by photon Monte Carlo
 * (radiate2, 4290-4372), its Poisson photon count and photon uniforms drawn
 * from the same per-particle generator. */
int stb_set_radiation(int radiate, unsigned long long seed);

/* Cal_SRLoss_U0rad (track_form 0) / Cal_SRLoss_U0rad_Track (track_form 1),
 * simtrack.cpp:20691-20766: the reference particle's synchrotron-radiation
 * loss per turn in MeV (also kept as GP.U0rad), 0 unless GP.radiate.  GSBENDs
 * (and, in the track form, every sector bend) take their path on the orbit
 * stored in the element before them (stb_cal_orbit fills it; zero before);
 * a bend as the line's first element is rejected (the reference would read
 * before the line).  Host computation, no GPU. */
int stb_cal_srloss_u0rad(stb_line *line, int track_form, double *u0rad_mev);
/* Cal_SRLoss_Particle, simtrack.cpp:20768-20781: x6 passed once through
 * every element of the line but the RF cavities, on `device`, and updated in
 * place; *loss_mev = (pt - pt0) * GP.beta * GP.energy.  Radiating bends draw
 * from particle 0's deviate stream at turn 0.  The reference passes without
 * loss tests; a particle that Track()'s tests would stop (|x| or |y| > 0.1 at
 * entry, outside an element's aperture, NaN) is rejected with STB_EINVAL and
 * x6 unchanged. */
int stb_cal_srloss_particle(stb_line *line, double *x6, double *loss_mev, int device);
/* out[0..7] = GP.gamma, GP.beta, GP.energy, GP.brho, GP.Q, GP.energy0, GP.G, GP.p */
int stb_get_ref(double *out8);

/* ---- elements: `new TYPE(name, args...)`  simtrack.h:399-1059 ----
 * type: "DRIFT","MARKER","SBEND","GSBEND","QUAD","SKEWQ","SEXT","OCT","MULT","GMULT",
 *       "SBENDMULT","KICKER","HKICKER","VKICKER","RFCAV","CRABRF","CCMULT","LBT","ILBT",
 *       "BEAMBEAM","BPM","HBPM","VBPM","SOLEN","PATCH".
 * args: the constructor arguments after `name`, in constructor order (SOLEN: L, KS;
 *       PATCH: DX, DY, DS, THETA, simtrack.cpp:9645, 12262); MULT takes
 *       L, KNL[11], KNSL[11] (23 values); GMULT/SBENDMULT take L, ANGLE, E1, E2,
 *       KNL[11], KNSL[11] (26 values); BEAMBEAM takes TREATMENT, NP, BBSCALE, SIGMAL,
 *       NSLICE, EMITX, BETAX, ALFAX, EMITY, BETAY, ALFAY. */
int stb_element_new(const char *type, const char *name, const double *args, int nargs, stb_element **out);
/* delete of an element that is not owned by a line */
int stb_element_free(stb_element *e);
/* Element::SetP / Element::GetP  (e.g. QUAD simtrack.cpp:8645-8685) */
int stb_element_setp(stb_element *e, const char *pname, double value);
int stb_element_getp(const stb_element *e, const char *pname, double *value);
/* public fields DX, DY, DS, DTHETA, DPHI, DPSI  (simtrack.h:388-389) */
int stb_element_set_misalign(stb_element *e, double dx, double dy, double ds, double dtheta, double dphi,
                             double dpsi);
/* public fields APx, APy  (simtrack.h:394; default 1 m, simtrack.cpp:8394-8395) */
int stb_element_set_aperture(stb_element *e, double apx, double apy);
/* writes NAME into buf (NUL-terminated, truncated to cap) */
int stb_element_name(const stb_element *e, char *buf, int cap);
/* out[0..9] = public fields L, S, DX, DY, DS, DTHETA, DPHI, DPSI, APx, APy (simtrack.h:384-394) */
int stb_element_geometry(const stb_element *e, double *out10);
/* writes TYPE into buf (NUL-terminated, truncated to cap) */
int stb_element_type(const stb_element *e, char *buf, int cap);

/* ---- Line (simtrack.cpp:12341-12431); the line owns appended elements ---- */
int stb_line_new(stb_line **out);
int stb_line_free(stb_line *l);                       /* ~Line -> Empty() */
int stb_line_append(stb_line *l, stb_element *e);     /* Line::Append */
int stb_line_insert(stb_line *l, long i, stb_element *e); /* Line::Insert */
int stb_line_delete(stb_line *l, long i);             /* Line::Delete */
int stb_line_replace(stb_line *l, long i, stb_element *e); /* Line::Replace */
int stb_line_rewind(stb_line *l, long i);             /* Line::Rewind */
int stb_line_invert(stb_line *l);                     /* Line::Invert */
long stb_line_ncell(const stb_line *l);               /* Line::Ncell */
double stb_line_length(const stb_line *l);            /* Line::Length */
int stb_line_cell(stb_line *l, long i, stb_element **out); /* Line::Cell[i] (borrowed) */
/* Read_MADX_Lattice(line, filename), simtrack.cpp:13591-13791: appends the
 * elements of a MAD-X TFS twiss table (see include/simtrack_b200.hpp). */
int stb_line_read_madx(stb_line *l, const char *path);
/* Read_BMAD_Lattice(line, filename), simtrack.cpp:14054-14244: appends the
 * elements of a Bmad lattice table (see include/simtrack_b200.hpp). */
int stb_line_read_bmad(stb_line *l, const char *path);

/* ---- flattening: Line -> device element table ----
 * No reference counterpart: the reference dispatches Element::Pass virtually
 * per particle per element (simtrack.cpp:20801).  The table snapshots GP and
 * every element parameter; rebuild it after editing the line. */
int stb_table_create(const stb_line *l, int device, stb_table **out);
int stb_table_free(stb_table *t);
/* info[0] = elements, [1] = pool doubles, [2] = algorithmic FP64 ops per particle-turn,
 * [3] = 1 if the current launch variant stages the table in shared memory,
 * [4] = table bytes (shared memory per CTA when staged), [5] = launch variant */
int stb_table_info(const stb_table *t, double *info6);

/* Autotuner (no reference counterpart): times every launch variant of the
 * tracking kernel (CTA size, registers per thread, table in shared memory or
 * L1) on a device-side copy of the n given particles for nturn turns and keeps
 * the fastest for this table.  The inputs are not modified.  timings_ms
 * (optional) receives up to ntimings per-variant times (< 0: not runnable). */
int stb_table_autotune(stb_table *t, const double *x, const double *px, const double *y, const double *py,
                       const double *z, const double *pt, long n, int nturn, double aperture_radius, int *chosen,
                       double *timings_ms, int ntimings);
int stb_table_set_variant(stb_table *t, int variant);
/* The autotuner for a spin table (stb_table_create_spin): xs9 = the nine
 * device arrays x, px, y, py, z, pt, sx, sy, sz of n particles (not
 * modified); chooses among the spin kernel's launch variants, whose names
 * stb_spin_variant_info gives.  stb_table_set_variant indexes the spin
 * variants for a spin table. */
int stb_table_autotune_spin(stb_table *t, const double *const *xs9, long n, int nturn, double aperture_radius,
                            int *chosen, double *timings_ms, int ntimings);
int stb_spin_variant_info(int variant, char *name, int cap, int *block, int *smem);
/* Contraction policy of the table's tracking kernel (no reference
 * counterpart).  fast = 0 (default): the strict kernel, in which every FP64
 * add and multiply rounds separately as in the reference's x86-64 build, so
 * results equal the reference's.  fast != 0: the same kernel compiled with
 * FMA contraction; each contracted multiply-add rounds once, so coordinates
 * differ from the reference's in the last bits and chaotic trajectories
 * separate over many turns.  Applies to stb_track_device / stb_track_host
 * and the autotuner on this table. */
int stb_table_set_contraction(stb_table *t, int fast);
/* Segmented staging (no reference counterpart).  An orbit table too large to
 * sit in shared memory whole is cut into consecutive segments of at most
 * `bytes` bytes each (element headers plus their parameters); the seg_*
 * launch variants stage them into two shared-memory buffers with bulk copies,
 * the next segment's copy running while the current one is tracked.  The
 * autotuner picks the segment size; stb_table_set_segment_bytes sets it
 * (1024 bytes to half the shared memory of a CTA; STB_EINVAL for tables that
 * fit whole and spin tables).  stb_table_segments reports the current plan
 * (nseg = 0: none). */
int stb_table_set_segment_bytes(stb_table *t, long bytes);
int stb_table_segments(const stb_table *t, int *nseg, int *seg_bytes);
/* name (NUL-terminated, truncated to cap), CTA size and shared-memory flag of a launch variant */
int stb_track_variant_info(int variant, char *name, int cap, int *block, int *smem);

/* ---- tracking ----
 * Track()  simtrack.cpp:20791-20814, batched.  Coordinates are SoA device
 * arrays of n doubles each (x, px, y, py, z=-c*dt, pt=dE/P0c; simtrack.cpp:12-21),
 * updated in place.  lost_turn[i] < 0 marks a live particle on entry and exit;
 * a lost particle gets the turn (turn0-based global index) and the element
 * index after which it was lost, and keeps its coordinates at that point, as
 * in the reference.  turn0 == 0 applies Track()'s entry check
 * (|x| or |y| > 0.1 m -> lost at turn 0, element 0).  aperture_radius > 0 adds
 * the circular loss test x^2 + y^2 > R^2 after every element.
 * stream: a cudaStream_t, or NULL for the default stream.  Asynchronous. */
int stb_track_device(stb_table *t, double *x, double *px, double *y, double *py, double *z, double *pt, long n,
                     int turn0, int nturn, double aperture_radius, int32_t *lost_turn, int32_t *lost_elem,
                     void *stream);

/* Host-buffer form with Track()'s outputs: x is AoS n*6 (x[6] per particle as in
 * Track), stable[i] on entry is Track()'s input flag (0 -> lost immediately);
 * on exit stable/lost_turn/lost_post hold Track()'s outputs.  Copies in and
 * out, synchronous. */
int stb_track_host(stb_table *t, double *x, long n, int nturn, double aperture_radius, int *stable,
                   int *lost_turn, int *lost_post);

/* Seed-batched tracking that allocates nothing (no counterpart in the
 * reference).  Same semantics as stb_track_device applied to each table in
 * turn: nseed tables (one device, one reference particle), seed s owning
 * n_per_seed[s] consecutive particles of the SoA device arrays x..pt,
 * lost_turn, lost_elem; particles with lost_turn >= 0 on entry are skipped.
 * Its work list, counters and status word live in a fixed static device
 * array sized for at most STB_STATIC_MAX_SEEDS seeds and
 * STB_STATIC_MAX_PARTICLES particles in total (larger requests fail with
 * STB_EINVAL): for callers whose device memory belongs to another allocator's
 * pool, or which must not call cudaMalloc/cudaFree (they synchronise the
 * device) between their own kernels.  Each call rewrites the whole scratch
 * before use; every call looks the scratch up (cudaGetSymbolAddress,
 * no allocation).  Never call it while `stream` or its device is being
 * captured into a CUDA graph: it copies its status word back and waits for
 * `stream` before returning.  Calls that overlap in time on one device race
 * on the shared scratch.  Tables are handles of one CUDA context: after
 * cudaDeviceReset they may not be used again. */
#define STB_STATIC_MAX_SEEDS 64
#define STB_STATIC_MAX_PARTICLES 1048576
int stb_track_seeds_static(stb_table *const *tables, int nseed, const long *n_per_seed, double *x, double *px,
                           double *y, double *py, double *z, double *pt, int32_t *lost_turn, int32_t *lost_elem,
                           int turn0, int nturn, double aperture_radius, void *stream);

/* Cal_Orbit_Num(line, deltap), simtrack.cpp:14947-15030: 4D closed orbit at
 * momentum offset deltap (Newton iteration on the GPU one-turn map, RF off);
 * stores each element's X[] and, when orbit6 is not NULL, writes the orbit
 * after element j to orbit6[j*6 + k]. */
int stb_cal_orbit(stb_line *l, double deltap, double *orbit6, int device);

/* Track_DA(line, nturn, deltap0, sigmax0, sigmay0, filename), simtrack.cpp:21389-21441:
 * the stable amplitude of 10 phase angles by twin-particle bisection, written
 * to filename as the reference writes it (NULL: no file) and returned in
 * angles10 / sigma10 (optional).  All reachable bisection midpoints are
 * tracked in one batched launch, then the bisections are replayed. */
int stb_track_da(stb_line *l, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
                 double *angles10, double *sigma10, int device);

/* The reference's other DA drivers with their output files (see
 * include/simtrack_b200.hpp):
 *   STB_DA1 Track_DA1 (simtrack.cpp:21443), STB_DA2 Track_DA2 (21497),
 *   STB_DA3 Track_DA3 (21535), STB_DA_RADIAL Track_DA_Radial (21682):
 *     bisections; out_a / out_sigma (optional, 10 entries) receive the angle
 *     labels [deg] and stable amplitudes, *nout their number (5 or 10);
 *   STB_DA_UNIFORM Track_DA_Uniform (21574), STB_DA_RADIAL_UNIFORM
 *     Track_DA_Radial_Uniform (21736): a sweep at `angle` [rad]; out_a /
 *     out_sigma (optional, 150 entries) receive each written line's stable
 *     flag (1.0 / 0.0) and amplitude, *nout the number of lines (up to the
 *     first loss, where the reference ends the process).
 * `angle` is ignored by the bisections; filename may be NULL. */
#define STB_DA1 1
#define STB_DA2 2
#define STB_DA3 3
#define STB_DA_RADIAL 4
#define STB_DA_UNIFORM 5
#define STB_DA_RADIAL_UNIFORM 6
int stb_track_da_driver(stb_line *l, int which, int nturn, double deltap0, double angle, double sigmax0,
                        double sigmay0, const char *filename, double *out_a, double *out_sigma, long *nout,
                        int device);

/* Cal_Tunes_Track (simtrack.cpp:20971-20990): x6 (in/out) tracked nturn turns
 * with a turn-by-turn record (x[0], x[2] below 1e-9 raised by 1e-9 first);
 * if it survives, tunes2 = FineTuneFinder of its x and y records in
 * [tune_lower, tune_upper) and *stable = 1, else tunes2 is left alone and
 * *stable = 0. */
int stb_cal_tunes_track(stb_line *l, double *x6, int nturn, double tune_lower, double tune_upper, double *tunes2,
                        int *stable, int device);
/* Cal_Tunes_Track(line, deltap0) (simtrack.cpp:20992-21025): the tunes of the
 * closed orbit at deltap0 over 1,024 turns (line.Tune1/Tune2; 0 if lost). */
int stb_cal_tunes_track_orbit(stb_line *l, double deltap0, double tune_lower, double tune_upper, double *tunes2,
                              int device);
/* Cal_Chrom_Track (simtrack.cpp:21027-21051): chroms4 = Chromx1, Chromy1,
 * Chromx2, Chromy2 from the tracked tunes at deltap = +3e-4, -3e-4, 0.
 * stb_cal_tunes_track, stb_cal_tunes_track_orbit and stb_cal_chrom_track set
 * the process-wide tune window (the reference's globals tune_low, tune_high)
 * for the length of the call: do not call them from two host threads at
 * once. */
int stb_cal_chrom_track(stb_line *l, double tune_lower, double tune_upper, double *chroms4, int device);

/* ---- Track_Radial (simtrack.cpp:21641-21680) ----
 * As stb_track_device / stb_track_host, with z corrected after every element
 * j by the path-length change of the on-momentum reference particle through
 * j (x04[j], from a particle started at zero with z and pt reset before each
 * element, simtrack.cpp:21652-21657).  The first call on a table computes
 * x04 on the device (allocation and a synchronisation); later calls reuse it. */
int stb_track_radial_device(stb_table *t, double *x, double *px, double *y, double *py, double *z, double *pt,
                            long n, int turn0, int nturn, double aperture_radius, int32_t *lost_turn,
                            int32_t *lost_elem, void *stream);
int stb_track_radial_host(stb_table *t, double *x, long n, int nturn, double aperture_radius, int *stable,
                          int *lost_turn, int *lost_post);
/* Cal_dz0_OnMomentumPart (simtrack.cpp:20929-20940): x0[6] (host, in/out)
 * through every element with z and pt reset before each; dz0 (host, ncell)
 * receives its z after each element. */
int stb_cal_dz0(stb_line *l, double *x0, double *dz0, int device);
/* Track_wrt_OnMomentumPart (simtrack.cpp:20942-20967): as stb_track_radial_host
 * (no circular aperture) with the caller's dz0[ncell] in place of the
 * on-momentum path. */
int stb_track_wrt_onmom(stb_line *l, double *x, long n, const double *dz0, int nturn, int *stable, int *lost_turn,
                        int *lost_post, int device);
/* Per-element probe of Track_Radial (layout as stb_track_probe). */
int stb_track_radial_probe(stb_table *t, double *x, long n, int nturn, double aperture_radius, double *dump,
                           int *stable, int *lost_turn, int *lost_post);

/* ---- spin tracking: Track_Spin (simtrack.cpp:21766-21789) ----
 * A spin table is flattened with Element::sPass semantics: orbit slices
 * interleaved with the Thomas-BMT rotation spin() (4574-4630) of
 * SBEND/QUAD/SKEWQ/SEXT/OCT/MULT/SBENDMULT/KICKER (7486-8208); CRABRF acts as
 * a drift and RF/CCMULT/LBT/ILBT/BEAMBEAM leave the spin unchanged, as the
 * reference's sPass does.  GSBEND and GMULT are rejected (STB_EUNSUPPORTED).
 * The spin G is the one set by stb_set_spin_g before the table is created.
 * Spin tables work only with the stb_track_spin_* entry points. */
int stb_table_create_spin(const stb_line *l, int device, stb_table **out);
/* Device SoA form: orbit arrays as stb_track_device plus the spin unit
 * vector (x[6], x[7], x[8] of the reference) in sx, sy, sz.  Asynchronous. */
int stb_track_spin_device(stb_table *t, double *x, double *px, double *y, double *py, double *z, double *pt,
                          double *sx, double *sy, double *sz, long n, int turn0, int nturn, double aperture_radius,
                          int32_t *lost_turn, int32_t *lost_elem, void *stream);
/* Host AoS x[n*9] form with Track_Spin()'s outputs.  Synchronous. */
int stb_track_spin_host(stb_table *t, double *x9, long n, int nturn, double aperture_radius, int *stable,
                        int *lost_turn, int *lost_post);
/* As stb_track_spin_host, also writing the nine coordinates after every
 * element to dump9[((i*nturn + turn)*ncell + j)*9 + k] (small n). */
int stb_track_spin_probe(stb_table *t, double *x9, long n, int nturn, double aperture_radius, double *dump9,
                         int *stable, int *lost_turn, int *lost_post);

/* Per-element probe: as stb_track_host, and additionally writes the six
 * coordinates after every element to dump[((i*nturn + turn)*ncell + j)*6 + k]
 * (host buffer of n*nturn*ncell*6 doubles; entries after a particle's loss are
 * left as passed in).  This is the commented-out per-element output of
 * Track(), simtrack.cpp:20806-20812, made available for parity checks and
 * diagnostics.  Intended for small n. */
int stb_track_probe(stb_table *t, double *x, long n, int nturn, double aperture_radius, double *dump, int *stable,
                    int *lost_turn, int *lost_post);

/* ---- batched dynamic-aperture scan ----
 * Replaces the per-particle loops of the DA drivers (Track_DA, simtrack.cpp:21389-21441;
 * Track_DA_Radial_Uniform, 21736-21764), which call Track() once per initial
 * condition: nseed lattices (one table per field-error seed, all flattened for
 * the same reference particle, all on `device`) x n_per_seed[s] initial
 * conditions each, given as one host AoS array x0 (seed 0's particles first).
 * The tables must outlive the scan.  Particles are tracked in turn blocks of
 * work list / tracking / compaction; Track()'s loss convention and entry
 * check apply, plus the circular aperture when aperture_radius > 0. */
int stb_scan_create(stb_table **tables, int nseed, const double *x0, const long *n_per_seed, double aperture_radius,
                    int device, stb_scan **out);
int stb_scan_free(stb_scan *s);
/* Launch variant of the scan's tracking kernel (< 0 keeps the current one) and
 * particles per work item (<= 0 keeps the current one; multiple of 32, >= 64). */
int stb_scan_configure(stb_scan *s, int variant, int chunk);
/* Advances all live particles by nturn turns (stops early when none is left),
 * turns_per_block turns between compactions; use_graph != 0 replays the turn
 * blocks from a captured CUDA graph.  Synchronous. */
int stb_scan_run(stb_scan *s, int nturn, int turns_per_block, int use_graph);
/* Per original particle (in x0 order): Track()'s lost turn (-1: still alive),
 * element index of the loss, and the coordinates (AoS, at the loss or now).
 * Any output pointer may be NULL. */
int stb_scan_results(stb_scan *s, int32_t *lost_turn, int32_t *lost_elem, double *x_aos);
/* Autotuner: times one turn block of nturn turns for every launch variant of
 * the scan's tracking kernel on a snapshot of the current state (restored
 * after each trial, so the scan does not advance) and keeps the fastest.
 * timings_ms (optional) receives up to ntimings times (< 0: not runnable). */
int stb_scan_autotune(stb_scan *s, int nturn, int *chosen, double *timings_ms, int ntimings);
/* st[0] turns done, [1] device milliseconds, [2] turn blocks, [3] variant, [4] chunk, [5] particles */
int stb_scan_stats(const stb_scan *s, double *st6);
/* Turn-by-turn record at the start of the line, as Track_tbt (simtrack.cpp:20841)
 * keeps it, for all particles at once: after global turn t < nturns the scan
 * writes x, px, y, py of particle i (x0 order) to tbt[(t*4 + k)*n + i], n the
 * scan's particle count; tbt is a device buffer of nturns*4*n doubles owned by
 * the caller (entries of lost particles stop at their loss).  nturns = 0
 * switches recording off. */
int stb_scan_set_tbt(stb_scan *s, double *tbt, int nturns);
/* Removes the live particles with mask[i] != 0 (host array of n bytes, x0
 * order) from further tracking; their result is lost_turn = STB_RETIRED with
 * the coordinates at retirement.  Used by the surrogate to stop tracking the
 * particles it has classified. */
#define STB_RETIRED 0x40000000
int stb_scan_retire(stb_scan *s, const uint8_t *mask);
/* Stopping and resuming long scans (the reference's Track_DA* loops have
 * neither; a 1e5-turn scan of many seeds runs for many minutes).
 * stb_scan_set_abort(s, 1), callable from any host thread while another one
 * is inside stb_scan_run, sets a flag in mapped host memory that every turn
 * block reads on the device: the blocks still queued track nothing, and
 * stb_scan_run returns STB_EABORTED at a turn-block boundary with the state
 * intact.  While the flag is set every stb_scan_run returns STB_EABORTED at
 * once; stb_scan_set_abort(s, 0) re-arms the scan. */
int stb_scan_set_abort(stb_scan *s, int value);
/* Work-item packing (no reference counterpart): 0 spreads the live particles
 * over every resident CTA in items down to one warp; 1 keeps every item at
 * the full chunk, so a small population runs on few SMs with many warps each.
 * stb_scan_autotune tries both with every launch variant and keeps the
 * faster; stb_scan_packing reports the current choice. */
int stb_scan_set_packing(stb_scan *s, int pack);
int stb_scan_packing(const stb_scan *s, int *pack);
/* Wall-clock budget of each stb_scan_run call in seconds (0: none), checked
 * between groups of turn blocks; when it is spent the call returns
 * STB_ETIMEOUT at a turn-block boundary with the state intact. */
int stb_scan_set_budget(stb_scan *s, double max_seconds);
/* Writes the scan's state (particle slots, ids, loss state, live counts, turn
 * counter, outputs) to `path` (through a temporary file renamed into place);
 * stb_scan_restore loads it into a scan created with the same tables and
 * particle counts (STB_EINVAL otherwise).  A restored scan continues exactly
 * as the saved one would have: results equal those of an uninterrupted run. */
int stb_scan_checkpoint(stb_scan *s, const char *path);
int stb_scan_restore(stb_scan *s, const char *path);

/* ---- turn-by-turn diagnostics ----
 * Track_tbt (simtrack.cpp:20841-20860) for n particles on the GPU: x AoS
 * n*6 (in/out), stable[] Track()'s input flags and outputs as in
 * stb_track_host; x_tbt[(i*nturn + turn)*6 + k] = coordinate k of particle i
 * at the start of each turn up to and including the turn of its loss
 * (nothing for particles rejected by the entry check); x_tbt may be NULL. */
int stb_track_tbt(stb_line *l, double *x, long n, int nturn, double *x_tbt, int *stable, int *lost_turn,
                  int *lost_post, int device);
/* Track_tbt with a BPM index (simtrack.cpp:20884-20905): as stb_track_tbt,
 * recording x[6] after element bpm_index in every turn that reaches it; the
 * per-element probe it runs needs n * ncell * 48 B < 4 GB (else STB_EINVAL). */
int stb_track_tbt_bpm(stb_line *l, double *x, long n, int nturn, double *x_tbt, int bpm_index, int *stable,
                      int *lost_turn, int *lost_post, int device);
/* Track_tbt_spin (simtrack.cpp:20863-20882): as stb_track_tbt with spin
 * tracking (Element::sPass), x AoS n*9 and x_tbt[(i*nturn + turn)*9 + k]. */
int stb_track_tbt_spin(stb_line *l, double *x9, long n, int nturn, double *x_tbt9, int *stable, int *lost_turn,
                       int *lost_post, int device);
/* Track_tbt_spin with a BPM index (simtrack.cpp:20907-20927): as
 * stb_track_tbt_bpm with spin tracking and nine coordinates (n * ncell * 72 B
 * < 4 GB). */
int stb_track_tbt_spin_bpm(stb_line *l, double *x9, long n, int nturn, double *x_tbt9, int bpm_index, int *stable,
                           int *lost_turn, int *lost_post, int device);
/* Track_tbt_FMA (simtrack.cpp:21179-21241) with FineTuneFinder's window
 * [tune_lower, tune_upper) (the reference's globals tune_low/tune_high):
 * writes the reference's FMA-output.dat rows to `filename`; *rows = their
 * number (may be NULL). */
int stb_track_tbt_fma(stb_line *l, double deltap0, double sigmax0, double sigmay0, double tune_lower,
                      double tune_upper, const char *filename, long *rows, int device);
/* Track_tbt_Lyapunov (simtrack.cpp:21243-21306): writes the reference's
 * Lmap-output.dat rows to `filename`; *rows = their number (may be NULL). */
int stb_track_tbt_lyapunov(stb_line *l, double deltap0, double sigmax0, double sigmay0, const char *filename,
                           long *rows, int device);
/* FineTuneFinder (simtrack.cpp:2288-2319; with px != NULL the x/px form,
 * 2321-2352) for nsig signals at once: sample i of signal j is
 * x[i*stride + j] (device arrays; stride >= nsig when nsig > 1), n <= 4096
 * samples; the same coarse 1e-3 scan over [tune_lower, tune_upper) and
 * ten-fold zooms down to a 1e-12 step.  tune: device array [nsig].
 * Asynchronous on `stream`. */
int stb_fine_tune(const double *x, const double *px, int n, long nsig, long stride, double tune_lower,
                  double tune_upper, double *tune, int device, void *stream);
/* Early-turn features of the loss-prediction surrogate (no reference
 * counterpart; built from Track_tbt_FMA's ingredients, simtrack.cpp:21179-21241):
 * per particle i, from tbt[(t*4 + k)*ntot + i] (t < nturn; x, px, y, py),
 * the initial coordinates x0[k*ntot + i] (k < 6) and the window tunes
 * tunes[w*ntot + i] (Qx, Qy of the first window, Qx, Qy of the second):
 * features[i*12 + f] = amplitude_x, amplitude_y (sigma units), 1e3*pt,
 * atan2(amp_y, amp_x), the four tunes, log10|dQx|, log10|dQy|, log10 of the
 * action spread over the record relative to the initial action, and the
 * largest amplitude reached.  twiss6 (host) = beta_x, alpha_x, beta_y,
 * alpha_y, emit_x, emit_y at the record point.  Asynchronous on `stream`. */
int stb_tbt_features(const double *tbt, long ntot, int nturn, const double *x0, const double *tunes,
                     const double *twiss6, float *features, int device, void *stream);

/* ---- loss-prediction surrogate (no reference counterpart) ----
 * MLP nin -> hidden -> hidden -> hidden -> nout (GELU, softmax cross-entropy)
 * with FP32 master parameters, bf16 operands and FP32 accumulation on the
 * tcgen05 tensor cores.  nin, nout <= 16; hidden a multiple of 16, <= 256;
 * batches are multiples of 16 up to max_batch.  x, labels, weights and probs
 * are device pointers (x: [B x nin] FP32 row-major; labels: int32 class ids;
 * weights: optional per-sample FP32 weights; probs: [B x nout]).
 * Parameter layout (stb_mlp_get_params/set_params, FP32): for each layer l,
 * W_l [out x in] row-major then b_l [out]. */
int stb_mlp_create(int nin, int hidden, int nout, int max_batch, unsigned long long seed, int device, stb_mlp **out);
int stb_mlp_free(stb_mlp *m);
long stb_mlp_param_count(const stb_mlp *m);
/* which = 0: parameters, 1: gradients of the last stb_mlp_gradients/train_step */
int stb_mlp_get_params(stb_mlp *m, float *host, int which);
int stb_mlp_set_params(stb_mlp *m, const float *host);
int stb_mlp_set_adamw(stb_mlp *m, float lr, float beta1, float beta2, float eps, float weight_decay);
int stb_mlp_forward(stb_mlp *m, const float *x, int B, float *probs);
/* Loss (host, may be NULL) and gradients of the weighted mean cross-entropy, no update. */
int stb_mlp_gradients(stb_mlp *m, const float *x, const int32_t *labels, const float *weights, int B, float *loss);
/* Gradients, then one AdamW step (decoupled weight decay, bias-corrected moments). */
int stb_mlp_train_step(stb_mlp *m, const float *x, const int32_t *labels, const float *weights, int B, float *loss);
/* Diagnostics: C[M x N] (FP32, row stride ldc) = A[M x K] * B[N x K]^T for bf16 device
 * matrices through the tcgen05 GEMM kernel (N a multiple of 16 <= 256, K of 16). */
int stb_mlp_gemm_test(const void *A, int lda, const void *B, int ldb, int M, int N, int K, float *C, int ldc,
                      int device);

/* Diagnostics (no reference counterpart): evaluates the kernels' elementary
 * functions on host buffers, on GPU `device` (device >= 0) or on the host CPU
 * (device < 0).  fn: 0 asin, 1 exp, 2 sin, 3 cos, 4 integer power (input pairs
 * h, m), 5 quotient a/b through the shared-reciprocal correction (pairs a, b;
 * IEEE division on the host) as used by the tracking maps; 10..15 the same
 * through CUDA's / the C library's own functions and the IEEE division.
 * in has n values (2n for the two-argument functions). */
int stb_math_eval(int fn, const double *in, double *out, long n, int device);

/* Diagnostics: measured FP64 FMA throughput of `device` in TFLOP/s (8 independent
 * FMA chains per thread on every SM; the roofline denominator of the tracking kernel). */
int stb_fp64_peak(int device, double *tflops);

/* Diagnostics: the drift's square root, reciprocal and quotients as the
 * tracking kernels compute them (from the cached reciprocal of 1+delta, no
 * IEEE division or sqrt sequence) against IEEE sqrt and division, over n
 * random drift arguments drawn from `seed`, on GPU `device` or on the host
 * (device < 0).  mismatch4 receives the counts for pz, 1/pz, betaz, L/betaz. */
int stb_check_drift_quotients(long n, unsigned long long seed, int device, unsigned long long *mismatch4);

/* Diagnostics: the table-driven fast path of the tracking maps' correctly
 * rounded sin and cos against their double-double series, over n random
 * arguments drawn from `seed` (|x| < 800: log-uniform magnitudes, spin
 * rotation angles, and small offsets from multiples of pi/128), on GPU
 * `device` or on the host (device < 0).  count4 receives: sin results that
 * differ, cos results that differ, arguments left to the series among the
 * generic classes, and among the offsets from multiples of pi/128. */
int stb_check_sincos(long n, unsigned long long seed, int device, unsigned long long *count4);

/* Strong-strong beam-beam, soft-Gaussian 4D: BeamBeam4D_SoftGaussian(Np1,
 * Npart_1, PartDist_1, Np2, Npart_2, PartDist_2, gamma1, gamma2, bbscale1,
 * bbscale2), simtrack.cpp:22846-22872 (simtrack.h:1403).  Each beam's
 * transverse centroid and rms size (Cal_Mean_RMS, 724-743, its running sums
 * in particle order) kick the other beam's macro-particles through BB4D;
 * px and py of both AoS beams x1[6*n1], x2[6*n2] are updated in place.  The
 * _device form takes device arrays and is asynchronous on `stream` (one
 * collision at a time per device: the moments live in one static device
 * buffer); the _host form takes host arrays and returns when done. */
int stb_bb4d_soft_gaussian_device(double Np1, long n1, double *x1, double Np2, long n2, double *x2, double gamma1,
                                  double gamma2, double bbscale1, double bbscale2, int device, void *stream);
int stb_bb4d_soft_gaussian_host(double Np1, long n1, double *x1, double Np2, long n2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int device);

/* Strong-strong beam-beam by particle-in-cell, 4D: BeamBeam4D_PIC(Np1, Mp1,
 * xc1, Np2, Mp2, xc2, gamma1, gamma2, bbscale1, bbscale2),
 * simtrack.cpp:23286-23378 (simtrack.h:1407).  Each beam's charge, deposited
 * on a 64 x 64 grid 15 rms sizes wide around its centroid (the smaller rms
 * size of the two beams per plane), gives the potential through the
 * integrated Green function and FFT convolution on the doubled grid; the
 * field kicks the other beam's macro-particles within 29 cells of their own
 * centroid.  px and py of both AoS beams x1[6*n1], x2[6*n2] are updated in
 * place, equal to the reference's bit for bit.  Each beam needs at least two
 * macro-particles (an rms size), at most INT32_MAX / 9; a particle that
 * would fall outside the grid (non-finite coordinates or rms size) gives
 * STB_EINVAL.  Both forms return when done (the Green function is tabulated
 * on the host between the moments and the deposition); the _device form
 * works on device arrays on `stream`. */
int stb_bb4d_pic_device(double Np1, long n1, double *x1, double Np2, long n2, double *x2, double gamma1,
                        double gamma2, double bbscale1, double bbscale2, int device, void *stream);
int stb_bb4d_pic_host(double Np1, long n1, double *x1, double Np2, long n2, double *x2, double gamma1, double gamma2,
                      double bbscale1, double bbscale2, int device);

/* BeamBeam6D_PIC(Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2, bbscale1,
 * bbscale2, Nslice1, Nslice2), simtrack.cpp:23380-23615: the sliced 6D
 * collision of stb_bb6d_soft_gaussian_* (bunches reordered in place by z,
 * largest first; slices of Mp/Nslice particles; slice pairs in the
 * reference's collision order, each drifted to its collision point) with
 * each slice pair colliding as stb_bb4d_pic_* with N/Nslice; bit for bit.
 * Arguments as for stb_bb6d_soft_gaussian_*.  The reference also writes
 * every bunch and slice to ./bunch*.dat on each call; this build writes
 * nothing.  Both forms return when done. */
int stb_bb6d_pic_device(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                        double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2, int device,
                        void *stream);
int stb_bb6d_pic_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                      double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2, int device);

/* Lumi_Cal_PIC_6D_Angle(Np1, Mp1, Np2, Mp2, theta, Nslice1, Nslice2, x1, x2,
 * gamma1, gamma2, bbscale1, bbscale2, Ncoll, freq), simtrack.cpp:
 * 23946-24224: both bunches boosted to the head-on frame of half crossing
 * angle theta (Lorentz_Transfer, 6790-6815; they are returned boosted, as
 * the reference leaves them), then stb_lumi_pic_6d_host; bit for bit.
 * |theta| < 1.5.  The reference's bunch, slice and collision-order files are
 * not written. */
int stb_lumi_pic_6d_angle_host(double Np1, long Mp1, double Np2, long Mp2, double theta, int nslice1, int nslice2,
                               double *x1, double *x2, double gamma1, double gamma2, double bbscale1,
                               double bbscale2, int Ncoll, double freq, int device, double *lumi);

/* BeamBeam6D_PIC_NonOffset(Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2,
 * bbscale1, bbscale2, Nslice1, Nslice2, zb1, zb2, Nx, Ny, hx, hy, grn_c_r,
 * grn_c_i), simtrack.cpp:24282-24432: the slice-boundary driver of
 * stb_bb6d_soft_gaussian_zb_host (slices zb[s+1] <= z < zb[s], particles
 * kept in place, the same checks) with each slice pair colliding as
 * stb_bb4d_pic_nonoffset_* with N scaled by the slice's share; bit for bit.
 * Grid and Green spectrum (host arrays) as for stb_bb4d_pic_nonoffset_host. */
int stb_bb6d_pic_nonoffset_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2,
                                const double *zb1, const double *zb2, int Nx, int Ny, double hx, double hy,
                                const double *grn_c_r, const double *grn_c_i, int device);

/* BeamBeam6D_PIC_Interpolation(Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2,
 * bbscale1, bbscale2, Nslice1, Nslice2, zb1, zb2, Nx, Ny, hx, hy, grn_c_r,
 * grn_c_i), simtrack.cpp:24434-24700: slices and checks as for
 * stb_bb6d_pic_nonoffset_host; in each slice pair each slice in turn
 * deposits its charge drifted to the front and the back of the other slice
 * (two potentials), and the other slice's particles, each drifted to its
 * own collision point, take the field of the potential interpolated between
 * the two (Interpolate_Electric_Field_2Potential, 3096-3152), with N/Mp of
 * the whole depositing bunch; bit for bit. */
int stb_bb6d_pic_interpolation_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2,
                                    double gamma1, double gamma2, double bbscale1, double bbscale2, int nslice1,
                                    int nslice2, const double *zb1, const double *zb2, int Nx, int Ny, double hx,
                                    double hy, const double *grn_c_r, const double *grn_c_i, int device);

/* Lumi_Cal_PIC_6D(Np1, Mp1, Np2, Mp2, Nslice1, Nslice2, x1, x2, gamma1,
 * gamma2, bbscale1, bbscale2, Ncoll, freq), simtrack.cpp:23703-23944: the
 * sliced driver of stb_bb6d_pic_* (bunches reordered by z in place, slice
 * pairs in collision order, drifted to their collision points); per pair the
 * luminosity of stb_lumi_pic_4d_* with N/Nslice is summed into *lumi, then
 * the pair collides as soft Gaussians (BB4D, N/Nslice) and drifts back, so
 * px and py change too; bit for bit.  Slice arguments as for
 * stb_bb6d_soft_gaussian_*.  The reference also writes the collision order
 * to ./collide_order.dat; this build writes nothing. */
int stb_lumi_pic_6d_device(double Np1, long Mp1, double Np2, long Mp2, int nslice1, int nslice2, double *x1,
                           double *x2, double gamma1, double gamma2, double bbscale1, double bbscale2, int Ncoll,
                           double freq, int device, void *stream, double *lumi);
int stb_lumi_pic_6d_host(double Np1, long Mp1, double Np2, long Mp2, int nslice1, int nslice2, double *x1,
                         double *x2, double gamma1, double gamma2, double bbscale1, double bbscale2, int Ncoll,
                         double freq, int device, double *lumi);

/* Cal_Effective_Green_Function(xoffset, yoffset, Nx, Ny, hx, hy, grn_c_r,
 * grn_c_i), simtrack.cpp:2881-2921: the integrated Green function of the 2D
 * Poisson equation on the doubled 2Nx x 2Ny grid, transformed by the
 * reference's FFT2D, into host arrays of 4 Nx Ny doubles, bit for bit.  The
 * grid must be square with Nx a power of two from 8 to 512 (STB_EINVAL
 * otherwise; the reference's FFT2D assumes both).  Tabulated on the host,
 * transformed on `device`. */
int stb_pic_green_function(double xoffset, double yoffset, int Nx, int Ny, double hx, double hy, double *grn_c_r,
                           double *grn_c_i, int device);

/* BeamBeam4D_PIC_NonOffset(Np1, Mp1, xc1, Np2, Mp2, xc2, gamma1, gamma2,
 * bbscale1, bbscale2, Nx, Ny, hx, hy, grn_c_r, grn_c_i),
 * simtrack.cpp:24226-24280: the PIC collision on the caller's grid centred on
 * the origin (spacing hx, hy; Green spectrum grn_c_r/grn_c_i of 4 Nx Ny from
 * stb_pic_green_function(0, 0, ...)), particles within Nx/2 - 3 cells of the
 * origin depositing and kicked; bit for bit.  Grids as for
 * stb_pic_green_function.  The _host form takes host beams and Green arrays,
 * the _device form device ones, on `stream`; both return when done. */
int stb_bb4d_pic_nonoffset_device(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                  double gamma2, double bbscale1, double bbscale2, int Nx, int Ny, double hx,
                                  double hy, const double *grn_c_r, const double *grn_c_i, int device, void *stream);
int stb_bb4d_pic_nonoffset_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int Nx, int Ny, double hx, double hy,
                                const double *grn_c_r, const double *grn_c_i, int device);

/* Lumi_Cal_PIC_4D(Np1, Mp1, Np2, Mp2, x1, x2, Ncoll, freq),
 * simtrack.cpp:23617-23701: both beams' charge on one 64 x 64 grid spanning
 * their joint x-y extent widened by 4 cells per side, *lumi = Ncoll *
 * sum(src1 src2) (Np1/Mp1) (Np2/Mp2) freq / hx / hy / 1e4, equal to the
 * reference's bit for bit.  Beams that span no area, or hold non-finite x or
 * y (for which the reference's grid indices are undefined), give
 * STB_EINVAL.  Both forms return when done; the _device form reads device
 * arrays on `stream`. */
int stb_lumi_pic_4d_device(double Np1, long Mp1, double Np2, long Mp2, const double *x1, const double *x2, int Ncoll,
                           double freq, int device, void *stream, double *lumi);
int stb_lumi_pic_4d_host(double Np1, long Mp1, double Np2, long Mp2, const double *x1, const double *x2, int Ncoll,
                         double freq, int device, double *lumi);

/* Strong-strong beam-beam, sliced soft-Gaussian 6D: BeamBeam6D_SoftGaussian(
 * Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2, bbscale1, bbscale2, Nslice1,
 * Nslice2), simtrack.cpp:22874-23132 (simtrack.h:1406).  Both AoS bunches are
 * reordered in place by z, largest first (equal z keep their order), cut
 * into Nslice slices of Mp/Nslice particles (the remainder is not collided);
 * the slice pairs collide in the reference's order, each drifting to its
 * collision point, kicking as soft Gaussians (BB4D with N/Nslice) and
 * drifting back.  Unlike the reference, no slice-centroid files are written.
 * Every slice needs at least two particles.  The _device form synchronises
 * `stream` (the pair order is decided on the host from the slice centroids);
 * one collision at a time per device. */
int stb_bb6d_soft_gaussian_device(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                  double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2,
                                  int device, void *stream);
int stb_bb6d_soft_gaussian_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2,
                                int device);

/* The overload with slice boundaries, BeamBeam6D_SoftGaussian(..., Nslice1,
 * Nslice2, zb1, zb2), simtrack.cpp:23134-23283 (simtrack.h:1409): slice s of
 * a bunch holds its particles with zb[s+1] <= z < zb[s] (zb: nslice + 1
 * decreasing host values); particles keep their places; each slice pair
 * collides as the 4D soft-Gaussian form with N scaled by the slice's share
 * of its bunch.  Defined (as in the reference) for Nslice1 == Nslice2 and
 * slices of 2 .. 2*Mp/Nslice particles; otherwise STB_EINVAL and the bunches
 * are unchanged.  Host AoS bunches, updated in place. */
int stb_bb6d_soft_gaussian_zb_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2,
                                   double gamma1, double gamma2, double bbscale1, double bbscale2, int nslice1,
                                   int nslice2, const double *zb1, const double *zb2, int device);

/* Diagnostics: deviates k0 .. k0+n-1 of particle `id`'s quantum-excitation
 * stream under `seed` (see stb_set_radiation), evaluated on GPU `device` or
 * on the host (device < 0); out is host memory. */
int stb_rad_normals(unsigned long long seed, unsigned long long id, unsigned long long k0, long n, double *out,
                    int device);

/* Diagnostics: one Philox4x32-10 block (the stream's generator), for its
 * published known-answer vectors. */
int stb_philox4x32_10(const unsigned int ctr[4], const unsigned int key[2], unsigned int out[4]);

#ifdef __cplusplus
}
#endif

#endif
