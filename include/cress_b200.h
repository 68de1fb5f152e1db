/*
 * cress_b200 — C-ABI of the B200 (sm_100a) implementation of CReSS's solver
 * time integration.
 *
 * Boundary.  In the reference every hot-path routine is a Fortran module
 * procedure s_xxx(ids..., ni,nj,nk, arrays...) that resolves its options
 * from integer name-table ids (SrcOrig/getiname.f90) and works on
 * explicit-shape arrays a(0:ni+1, 0:nj+1, 1:nk) (e.g. SrcOrig/hevi.f90:106-160).
 * A Fortran shim (cress_b200/fortran/m_cress_gpu.f90, bind(C)) resolves the
 * ids once, then calls the entry points below with the VALUES and with the
 * Fortran arrays as plain float pointers in exactly that layout (x fastest,
 * halo 0..ni+1, 0..nj+1, k = 1..nk).  Nothing in these signatures is a
 * torch or C++ type.
 *
 * Ownership.  The library owns the device copy of the prognostic state
 * between calls; host arrays are only read or written inside the call that
 * receives them.  One context = one domain on one device, driven by one
 * host thread; contexts are not re-entrant.
 *
 * Errors.  Every entry point returns 0 on success or a CRESS_E_* code (the
 * reference has no return codes: it calls destroy(...,'stop') after a
 * collective chkerr, SrcOrig/chkerr_multi.f90; the shim maps nonzero to
 * that path).  cress_last_error() gives a one-line message.
 */
#ifndef CRESS_B200_H
#define CRESS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define CRESS_OK 0
#define CRESS_E_ARG 1
#define CRESS_E_UNSUPPORTED 2
#define CRESS_E_CUDA 3
#define CRESS_E_NONUNIFORM 4
#define CRESS_E_NONFINITE 5
#define CRESS_E_TIMEOUT 6
#define CRESS_E_STATE 7

/* Resolved namelist values (the reference reads them through
 * getiname/getrname; SrcOrig/rdconf.f90:88-146 lists the namelists). */
typedef struct cress_cfg {
  int ni, nj, nk;       /* array dims: ni = xdim = nx+3, nk = zdim (SrcOrig/setdim.f90:196-199) */
  float dx, dy, dz;     /* grid spacing; dz is the mean spacing when sthopt=1 */
  int sthopt;           /* 0 uniform, >=1 stretched vertical grid (jcb varies in k) */
  int impopt;           /* 1 = HE-VI (implicit vertical, Thomas solve), 0 = HE-VE (explicit) */
  int divopt;           /* divergence damping 0/1/2 (SrcOrig/pgrad.f90:260-349) */
  int buyopt;           /* 1 = buoyancy in the small step (SrcOrig/hevi.f90:377) */
  int gwmopt;           /* 0 only */
  float weicoe;         /* implicit weight beta (SrcOrig/advbspi.f90:140) */
  int wbc, ebc, sbc, nbc;  /* lateral BCs after chknlslv: -1 = periodic on all four sides, or
                              wbc = ebc = 4, 5 or 7 (open radiation x boundaries: phase speed per
                              point, its column average, or the constant gwave) with sbc = nbc = -1 */
  int bbc, tbc;         /* 2 = rigid (SrcOrig/vbcw.f90:201) */
  int tile;             /* HE-VI tile shape id (0 = default: 32x8, two rows per thread; 1-11 other shapes;
                           12, 13: 32x8 with the column kept on chip, FP64 throughout the solve, nk <= 68;
                           12 two rows per thread, 13 one) */
  /* large step (SrcOrig/forcedrv.f90:548-608, SrcOrig/timeflt.f90:335) */
  int advopt;           /* 2: 4th-order horizontal, 2nd-order vertical advection; 3: 4th order in z as well (periodic boundaries) */
  int smtopt;           /* 0 none, 2 horizontal, 3 horizontal + vertical 4th-order smoothing */
  int vspopt;           /* 0 none, 2 Rayleigh damping above botbar toward the base state */
  int coropt;           /* 0 none, 1 f-plane Coriolis on u, v */
  int tubopt;           /* 0 none, 1 Smagorinsky, 2 the 1.5-order TKE closure (isoopt=1, flat terrain,
                           no surface flux; SrcOrig/eddyvis.f90, SrcOrig/forcetke.f90) */
  int cphopt;           /* 0 dry, 3 cold-rain bulk (haiopt=0) */
  float smhcoe, smvcoe; /* smoothing coefficients */
  float filcoe;         /* Asselin filter coefficient */
  float fc;             /* 0.5*omega*sin(lat) (SrcOrig/trilat.f90:118-134) */
  char vspvar[16];      /* sponge switches u v w p pt qv q ... ('o' on / 'x' off) */
  float thresq;         /* mixing-ratio threshold of the microphysics (namelist thresq) */
  float gwave;          /* phase speed of the open boundaries, wbc = 7 (namelist gwave, m/s) */
  int reserved[6];
} cress_cfg;

typedef struct cress_ctx cress_ctx;

/* Fields addressed by the sync calls (CRESS_TKE, the turbulent kinetic
 * energy tke/tkep of the reference, exists with tubopt=2 only). */
enum cress_field {
  CRESS_U = 0, CRESS_V, CRESS_W, CRESS_PP, CRESS_PTP, CRESS_QV,
  CRESS_QC, CRESS_QR, CRESS_QI, CRESS_QS, CRESS_QG, CRESS_NI, CRESS_NS, CRESS_NG,
  CRESS_TKE, CRESS_NFIELD
};
/* Time levels: t-dt ("p" arrays: up, vp, ...), t (u, v, ...), t+dt ("f"). */
enum cress_level { CRESS_PAST = 0, CRESS_NOW = 1, CRESS_FUTURE = 2, CRESS_FORCING = 3 };

/* Base-state arrays in cress_set_base3d's list, in this order. */
enum cress_base {
  CRESS_B_JCB = 0, CRESS_B_JCB8U, CRESS_B_JCB8V, CRESS_B_JCB8W, CRESS_B_RBR, CRESS_B_PTBR,
  CRESS_B_RST, CRESS_B_RST8U, CRESS_B_RST8V, CRESS_B_RST8W, CRESS_B_RCSQ, CRESS_B_N
};

const char* cress_last_error(void);
int cress_abi_version(void);

/* Create a context on CUDA device `device` (the caller's rank's GPU).
 * Replaces the allocation of the solver arrays in SrcOrig/allocslv.f90:388
 * for the device side; the host arrays stay Fortran-owned. */
int cress_create(const cress_cfg* cfg, int device, cress_ctx** out);
void cress_destroy(cress_ctx* ctx);

/* Use an external CUDA stream (cudaStream_t passed as void*); NULL returns
 * to the context's own (non-blocking) stream.  All work of the context is
 * ordered on it. */
int cress_set_stream(cress_ctx* ctx, void* stream);
int cress_sync(cress_ctx* ctx);

/* Failure-path test hook, no counterpart in the reference: the number of
 * probes each ring wait of the HE-VI level loop (tile 0) makes before it
 * gives up (default 4194304; 0 gives up at once).  A wait that gives up
 * makes the kernel stop issuing copies, wait for the ones in flight and
 * return, and the next synchronizing call reports CRESS_E_TIMEOUT; the
 * context stays usable.  A negative value restores the default. */
int cress_set_spin_limit(cress_ctx* ctx, int probes);

/* Base state and metrics, as the reference holds them after s_inivar
 * (SrcOrig/inivar.f90:674-850: setbase, baserho, sndwave): CRESS_B_N host
 * arrays in reference layout.  They must be horizontally uniform (flat
 * terrain, no map factors); otherwise CRESS_E_NONUNIFORM. */
int cress_set_base3d(cress_ctx* ctx, const float* const* base3d);

/* The base state from a height-level sounding, computed on the device in
 * FP64: the hydrostatic integration of the sounding with its humidity
 * iteration (SrcOrig/set1d.f90:278-452, 536-540; vextlow.f90:150-220),
 * the interpolation to the scalar levels (intrpsnd.f90:190-230,
 * vint13.f90:120-170), base density and Exner function with the boundary
 * levels (setbase.f90:153-189, bcbase.f90:150-210), rho*J and its w-point
 * average (baserho.f90:150-160, var8uvw.f90:190-196, bc8w.f90:136,166) and
 * rho c^2 (sndwave.f90:119); replaces those routines for a horizontally
 * uniform grid.
 *   zph, jcb: nk+1 entries each (index k = 1..nk): w-level heights and
 *     the Jacobian of the column;
 *   sounding: 5 x nlev values, levels 1..nlev (heights increasing): z,
 *     u, v, theta (tvar = 'p') or temperature ('t'), and relative
 *     humidity in percent (hvar = 'r') or the mixing ratio (any other);
 *   psnd0: pressure at the lowest sounding level (Pa); thresq: mixing
 *     ratios at or below it become 0;
 *   columns (out): CRESS_BS_N columns of nk+1 doubles, in the order of
 *     enum cress_base_col; levels 1..nk-1 as the reference forms them,
 *     level nk repeating level nk-1 (rst8w: level nk-2, as bc8w).
 * CRESS_E_ARG when the integration reaches p <= 0 or the humidity does not
 * converge. */
enum cress_base_col {
  CRESS_BS_UBR = 0, CRESS_BS_VBR, CRESS_BS_PBR, CRESS_BS_PTBR, CRESS_BS_QVBR, CRESS_BS_RBR,
  CRESS_BS_PTVBR, CRESS_BS_PIBR, CRESS_BS_RST, CRESS_BS_RST8W, CRESS_BS_RCSQ, CRESS_BS_N
};
int cress_base_state(int nk, const double* zph, const double* jcb, int nlev, const double* sounding,
                     int tvar, int hvar, double psnd0, double thresq, double* columns, int device);

/* Host <-> device copy of one prognostic field at one time level
 * (reference layout).  Used at restart read / dump / restart write times
 * (SrcOrig/outres.f90:868-900 reads the same arrays).
 * cress_put_field is asynchronous on the context's stream: from pageable
 * host memory the data is taken before the call returns, but from
 * page-locked (pinned) memory the copy may still be running, so keep such a
 * buffer unchanged until the next synchronizing call (cress_sync,
 * cress_get_field, cress_diagnostics).  cress_get_field returns with the
 * data in `host`. */
int cress_put_field(cress_ctx* ctx, int field, int level, const float* host);
int cress_get_field(cress_ctx* ctx, int field, int level, float* host);

/* Asynchronous read-back of nfield fields of one time level into host
 * arrays (reference layout; page-locked memory for the copies to overlap):
 * the values are captured on the context's stream at this point of its
 * work, and the device->host copies run on a second stream, so they
 * overlap what the context does next (the next step's host->device copies
 * and compute).  Two read-backs may be in flight; a third first waits on
 * the device for the first.  cress_wait_fields returns once every
 * read-back issued so far has filled its host arrays, cress_wait_fields_to
 * once at most in_flight (0 or 1) of them are still running (the older
 * ones are filled); neither waits for the context's other work.  Both
 * return CRESS_E_TIMEOUT if a bounded device-side wait gave up in the work
 * before a completed read-back.  No counterpart in the reference (the dump
 * writer reads the same arrays, SrcOrig/outdmp3d.f90:159-169). */
int cress_get_fields_async(cress_ctx* ctx, int level, int nfield, const int* fields, float* const* host);
int cress_wait_fields(cress_ctx* ctx);
int cress_wait_fields_to(cress_ctx* ctx, int in_flight);

/* Asynchronous input of nfield distinct fields of one time level from host
 * arrays (reference layout; page-locked memory for the copies to overlap):
 * the host->device copies run on a stream of their own, so they overlap
 * the work the context already has queued (a previous step's compute and
 * read-back), and the values enter the level at this point of the
 * context's work, for the calls that follow.  Keep the host arrays
 * unchanged until a synchronizing call (cress_sync, cress_get_field,
 * cress_diagnostics) or a cress_wait_fields for a read-back issued after
 * this call returns.  No counterpart in the reference (its host arrays are
 * the state). */
int cress_put_fields_async(cress_ctx* ctx, int level, int nfield, const int* fields, const float* const* host);

/* Dump file records formed on the device: the 3-D history dump of one
 * time level as s_outdmp / s_outdmp3d write it for dmplev = 1 and
 * dmpfmt = 2 (SrcOrig/outdmp.f90:380-870, SrcOrig/outdmp3d.f90:159-238):
 * for each variable dmpvar selects, in s_outdmp's order, the records
 * k = 2..nk-2 of nx*ny native floats (i fastest), staggered variables
 * averaged to scalar points, 'o' adding the base state before the
 * perturbation (ubar, u, vbar, v, w, pbar, pp, ptbar, ptp, qvbar, qv), '-'
 * giving the total or the field alone (u, v, p, pt, qv), cold rain adding
 * qc qr qi qs qg (dmpvar(7:7)='o') and nci ncs ncg (dmpvar(8:8)='o'), the
 * TKE closure tke (dmpvar(12:12)='o').  The bytes are the .bin file.
 *   dmpvar: the namelist string (its first 16 characters are read);
 *   host null: only *nbytes and names are set (the size query);
 *   names (optional): the dumped variables, comma-separated.
 * pbar and p need the base pressure (cress_set_base_moist).  The maximum
 * wind (dmpvar(12:12) '+' or '-') is rejected with CRESS_E_UNSUPPORTED. */
int cress_dump_3d(cress_ctx* ctx, int level, const char* dmpvar, void* host, long long cap_bytes,
                  long long* nbytes, char* names, int names_cap);

/* Restart file records formed on the device: the records s_outres writes
 * after the base state (SrcOrig/outres.f90:903-1289) -- the present and
 * past levels of every prognostic field, the open-x phase speeds, the
 * surface precipitation planes and the TKE, each as a Fortran sequential
 * unformatted record (a 4-byte length before and after its payload; the
 * framing of gfortran and ifort below 2 GiB).  host null: size query.
 * cress_restart_read takes the same byte stream (the records s_rdres reads
 * back, SrcOrig/rdres.f90) and restores the device state; it checks every record's length first.
 * The y phase speeds the file carries are zero (periodic y). */
int cress_restart_write(cress_ctx* ctx, void* host, long long cap_bytes, long long* nbytes);
int cress_restart_read(cress_ctx* ctx, const void* host, long long nbytes);

/* y-slab decomposition of one domain over ranks, in place of the
 * reference's MPI halo exchange (SrcOrig/shiftsx.f90:139-205,
 * SrcOrig/sethalo.f90:485-505) and its allreduce of the sedimentation
 * sub-step (SrcOrig/chkfall.f90:88).  Each rank's context holds its slab
 * (nj = its rows + 3, the same ni, nk and base state as the others); y is
 * periodic over the ring of ranks (rank 0's southern neighbour is the last
 * rank), x periodic.  Once attached, cress_large_step exchanges the ghost
 * rows after every acoustic substep and at the end of the step, and the
 * sub-step minimum over all ranks, as the reference's ranks do; every rank
 * must step together.  Plain microphysics only; no CUDA graphs.
 *   cress_slab_attach_nccl: one rank per process and GPU, rows over NCCL
 *     (libnccl.so.2 loaded at run time); id: 128 bytes from
 *     cress_slab_nccl_id on one rank, passed to all.
 *   cress_slab_group_create / cress_slab_attach_local: the ranks are
 *     contexts of this process, each stepped by its own host thread; the
 *     rows move as device copies ordered by CUDA events and a host barrier
 *     (bounded: a rank that waits longer than the group's timeout, 60 s
 *     unless cress_slab_group_set_timeout says otherwise, returns
 *     CRESS_E_TIMEOUT, and every rank of a group with a failed rank
 *     returns CRESS_E_STATE).
 *   cress_slab_detach: back to a periodic single domain (between steps). */
typedef struct cress_slab_group cress_slab_group;
int cress_slab_group_create(int nranks, cress_slab_group** out);
void cress_slab_group_destroy(cress_slab_group* grp);
int cress_slab_group_set_timeout(cress_slab_group* grp, int ms);
int cress_slab_attach_local(cress_ctx* ctx, cress_slab_group* grp, int rank);
int cress_slab_nccl_id(void* id128);
int cress_slab_attach_nccl(cress_ctx* ctx, int rank, int nranks, const void* id128);
int cress_slab_detach(cress_ctx* ctx);

/* Acoustic small-step loop on the device-resident state: replaces the body
 * of s_smalldrv (SrcOrig/smalldrv.f90:343-398): future u, v, w, p' start
 * from the past level, then nsstp substeps of dts run with the forcing
 * level's u, v, w, p' forcings (ufrc, vfrc, wfrc, pfrc), HE-VI
 * (SrcOrig/hevi.f90:339-426) for impopt=1 or HE-VE (SrcOrig/heve.f90:
 * 337-406) for impopt=0.  The result is the FUTURE level. */
int cress_small_steps(cress_ctx* ctx, int nsstp, float dts);

/* Same call with host arrays, as s_smalldrv receives them: copies
 * up, vp, wp, ppp and the four forcings to the device, runs the loop,
 * copies uf, vf, wf, ppf back. */
int cress_smalldrv(cress_ctx* ctx, int nsstp, float dts,
                   const float* up, const float* vp, const float* wp, const float* ppp,
                   const float* ufrc, const float* vfrc, const float* wfrc, const float* pfrc,
                   float* uf, float* vf, float* wf, float* ppf);

/* Large-step base data beyond cress_set_base3d: the base winds ubr, vbr and
 * the Rayleigh coefficient rbct(:,:,:,2) of s_vspdmp (SrcOrig/vspdmp.f90:
 * 269-292), host arrays in reference layout (horizontally uniform), and
 * ksp0(2), the first damped level (SrcOrig/vspdmp.f90:222-232). */
int cress_set_base_large(cress_ctx* ctx, const float* ubr, const float* vbr, const float* rbct,
                         int ksp0);

/* One leapfrog large step on the device-resident state, replacing the body
 * of s_intgdrv for a dry run (SrcOrig/intgdrv.f90:866-1119 with s_fdmdrv,
 * SrcOrig/fdmdrv.f90:661-704): forcing of u, v, w, p', theta'
 * (s_forcedrv), nsstp HE-VI substeps of dts (s_smalldrv), the theta' step
 * (s_steps), the Asselin filter (s_timeflt), both periodic ghost planes
 * (bcycle, s_shift2nd) and the time-level rotation (s_swp2nxt).  ctime is
 * s_intgdrv's model time of the present level (ms); at ctime = 0 the
 * Asselin filter is skipped (SrcOrig/intgdrv.f90:968).  dtb and dts are
 * s_timeint's large and small steps (halves of dtbig, dtsml at ctime = 0,
 * SrcOrig/timeint.f90:160-190).  With cphopt=3 the step is the moist one:
 * moist buoyancy, the qv / species / number steps, s_cloudphy, the filter
 * of the moist fields and s_satadjst on t and t+dt
 * (SrcOrig/intgdrv.f90:832-998). */
int cress_large_step(cress_ctx* ctx, long long ctime, float dtb, int nsstp, float dts);

/* Domain diagnostics of one time level (level 0..2), in FP64 on the
 * device over the physical cells i = 2..ni-2, j = 2..nj-2, k = 2..nk-2:
 *   out[0] water of qv+qc+qr+qi+qs+qg, sum rst (q...) dx dy dz      (kg)
 *   out[1] precipitated water, sum of the accumulated surface
 *          precipitation of the five species times rhow dx dy       (kg)
 *   out[2] mass, sum rst (1 + p'/rcsq) dx dy dz                     (kg)
 *   out[3..6] max |u|, |v|, |w|, |theta'|
 *   out[7] number of non-finite values in the level's prognostic fields
 * (out[0..1] are 0 without microphysics).  Returns CRESS_E_NONFINITE when
 * out[7] > 0 (the blow-up detector; the reference's own monitor is the
 * max/min printout of SrcOrig/mxndrv.f90).  out holds 8 doubles. */
int cress_diagnostics(cress_ctx* ctx, int level, double* out);

/* Number of HE-VI tile shapes (cress_cfg.tile = 0 .. CRESS_NTILES-1). */
#define CRESS_NTILES 14

/* Autotuner: times every HE-VI tile shape (xy tile, ring depth, column
 * store) over `reps` small-step loops of nsstp substeps of length dts on
 * the current state, which it leaves untouched (only the future level is
 * written), and keeps the fastest as the context's tile.  best_tile and
 * ms_per_substep[CRESS_NTILES] (milliseconds per substep, -1 for shapes
 * this grid cannot use) may be null. */
int cress_autotune(cress_ctx* ctx, int nsstp, float dts, int reps, int* best_tile, float* ms_per_substep);

/* Ensembles.  An ensemble groups contexts of independent domains (any
 * sizes) on one device: cress_ensemble_large_step runs one large step of
 * every member, each as cress_large_step would, except that the acoustic
 * substeps of all members run as one kernel launch per substep over every
 * member's tiles (small domains fill the GPU together).  The rest of each
 * member's step stays on the member's own stream, so members overlap; the
 * shared launches run on the ensemble's stream, ordered against the
 * members' streams by events.  A step whose pointer states and parameters
 * were seen before replays one CUDA graph of the whole ensemble step
 * (cress_ensemble_set_graphs(e, 0) turns that off).  Members need impopt=1
 * and the same divopt, sthopt (zero or not) and buyopt.  The shared
 * acoustic launch runs tile 0's kernel or tile 13's (the FP64 right-hand
 * sides on chip; every member with 8 <= nk <= 68): tile 13 when every
 * member was created with tile 13, else tile 0, and the members are set
 * to the ensemble's tile.  cress_ensemble_set_tile switches it (0 or 13);
 * cress_ensemble_autotune times both over `reps` loops of nsstp batched
 * substeps of length dts on the members' present state (only the future
 * levels are written) and keeps the faster (best_tile, ms_per_substep[2]
 * for tiles 0 and 13, -1 where unusable; both may be null).  Members stay
 * valid contexts (sync calls, cress_large_step); destroy the ensemble
 * before its members. */
typedef struct cress_ensemble cress_ensemble;
int cress_ensemble_create(cress_ctx* const* members, int n, cress_ensemble** out);
void cress_ensemble_destroy(cress_ensemble* e);
int cress_ensemble_set_graphs(cress_ensemble* e, int on);
int cress_ensemble_set_tile(cress_ensemble* e, int tile);
int cress_ensemble_autotune(cress_ensemble* e, int nsstp, float dts, int reps, int* best_tile, float* ms_per_substep);
int cress_ensemble_large_step(cress_ensemble* e, long long ctime, float dtb, int nsstp, float dts);

/* Replay whole large steps from CUDA graphs (on != 0) instead of launching
 * every kernel from the host: the second step with a given time-level
 * state and parameters is captured, later ones launch the graph.  Results
 * are bitwise identical to the eager path. */
int cress_set_graphs(cress_ctx* ctx, int on);

/* Moist base state (cphopt=3): base pressure pbr and base water vapour qvbr
 * (SrcOrig/setbase.f90:153-189), host arrays in reference layout. */
int cress_set_base_moist(cress_ctx* ctx, const float* pbr, const float* qvbr);

/* Cold-rain bulk microphysics on the device-resident state, replacing
 * s_cloudphy for cphopt=3, haiopt=0 (SrcOrig/cloudphy.f90:277-466 ->
 * s_coldblk, SrcOrig/coldblk.f90:321-481): process rates from the PAST
 * level (theta', water species, ice numbers, p'), applied to the FUTURE
 * level, then sedimentation with the domain-global sub-step
 * (SrcOrig/fallblk.f90:298-543) accumulating surface precipitation.  dtb
 * is the leapfrog large step (the scheme integrates over 2*dtb).  thresq is
 * the namelist threshold of the mixing ratios. */
int cress_cloudphy(cress_ctx* ctx, float dtb, float thresq);

/* Saturation adjustment s_satadjst for cphopt=3 (SrcOrig/satadjst.f90:
 * 154-189: s_siadjst then s_swadjst) on one time level (CRESS_NOW or
 * CRESS_FUTURE) of theta', qv, qc, qi, ni, using that level's p'. */
int cress_satadjst(cress_ctx* ctx, int level, float thresq);

/* Surface precipitation planes prc, prr, pri, prs, prg, each as (rate,
 * accumulated) on the (ni+2) x (nj+2) plane: 10 planes, host layout. */
int cress_get_precip(cress_ctx* ctx, float* host);
int cress_put_precip(cress_ctx* ctx, const float* host);

/* Open x boundaries: the phase speeds of one variable (a cress_field),
 * host layout of the reference's ucpx(1:nj,1:nk,1:2) (west, east), as
 * s_phasev left them for the next large step (SrcOrig/phasev.f90; the
 * restart files carry them, SrcOrig/outrst.f90).  CRESS_E_STATE on a
 * periodic context. */
int cress_get_phase(cress_ctx* ctx, int field, float* host);
int cress_put_phase(cress_ctx* ctx, int field, const float* host);

/* Number of kernel launches the library issued since the context was
 * created (instrumentation for benchmarks). */
long long cress_launch_count(const cress_ctx* ctx);

/* ------------------------------------------------------------------------
 * Learned cold-rain microphysics.  No counterpart in the reference: a
 * per-cell MLP (16 inputs, 3 hidden layers of 256 with SiLU, 9 outputs;
 * BF16 weights and activations, FP32 accumulation on the tensor cores)
 * that replaces the process-rate part of s_coldblk (adjstni, srcblk,
 * adjstni: SrcOrig/coldblk.f90:327-425).  It is trained by the library's
 * own forward, backward and Adam kernels on tuples that the plain scheme
 * produces on the device; in use, positivity and water conservation are
 * enforced after inference, and cells outside the training envelope or
 * failing the water-budget residual check run the plain scheme.
 *
 * Inputs (per cell, before standardization): T-273.16, ln p, rho, w,
 * log10 of qv, qc, qr, qi, qs, qg (floor 1e-12), log10 of ni, ns, ng
 * (floor 1), supersaturation over water and over ice (clipped to [-1,1]),
 * log10 of the future level's total condensate.  Outputs: for the changes
 * d of qv, qc, qr, qi, qs, qg, ni, ns, ng over 2*dtb, y = sign(d) *
 * log10(1 + |d|/s) with s = 1e-9 (mixing ratios) or 1 (numbers).
 * Normalisation block (cress_mlp_get_norm, 82 floats): input means (16),
 * input scales (16), output means (9), output scales (9), input minimum
 * (16) and maximum (16) of the training set (the envelope).
 * Parameters (cress_mlp_param_count floats): W1 [256][64] (inputs padded
 * to 64), b1 [256], W2 [256][256], b2, W3 [256][256], b3 (W_l stored
 * [out][in]), W4 [256][64] ([in][out], outputs padded to 64), b4 [64].
 * ---------------------------------------------------------------------- */
typedef struct cress_mlp cress_mlp;

int cress_mlp_param_count(void);
int cress_mlp_create(int device, unsigned long long seed, cress_mlp** out);
void cress_mlp_destroy(cress_mlp* m);
int cress_mlp_get_params(cress_mlp* m, float* host);
int cress_mlp_set_params(cress_mlp* m, const float* host);
int cress_mlp_get_norm(cress_mlp* m, float* host);
int cress_mlp_set_norm(cress_mlp* m, const float* host);
/* Network function: x [n][16] standardized inputs -> y [n][9]. */
int cress_mlp_forward(cress_mlp* m, int n, const float* x, float* y);
/* Mean-square loss and its gradient w.r.t. every parameter for one batch
 * (x [n][16], t [n][9] standardized; n a multiple of 128). */
int cress_mlp_loss_grad(cress_mlp* m, int n, const float* x, const float* t, float* loss, float* grad);
/* Tuple store (transformed, unstandardized features and targets). */
int cress_mlp_reserve(cress_mlp* m, long long cap);
int cress_mlp_add_tuples(cress_mlp* m, long long n, const float* x, const float* t);
int cress_mlp_get_tuples(cress_mlp* m, long long first, long long n, float* x, float* t);
long long cress_mlp_tuple_count(const cress_mlp* m);
/* Normalisation and envelope from the stored tuples. */
int cress_mlp_fit_norm(cress_mlp* m);
/* `steps` Adam steps on random batches (batch % 128 == 0) of the store;
 * losses (may be NULL) receives each step's loss. */
int cress_mlp_train(cress_mlp* m, int steps, int batch, float lr, unsigned long long seed, float* losses);
/* Use the MLP for the process rates in the context's s_cloudphy (NULL
 * returns to the plain scheme).  chunk 0: one fused persistent kernel over
 * all cells (activations stay on chip); chunk > 0: batches of that many
 * cells through separate GEMM launches.  resid_tol: relative tolerance of
 * the water-budget residual. */
int cress_set_learned_micro(cress_ctx* ctx, cress_mlp* m, int chunk, float resid_tol);
int cress_learned_stats(cress_ctx* ctx, long long* mlp_cells, long long* fallback_cells);
/* Sample training tuples of the plain scheme on every following
 * s_cloudphy into the MLP's store (up to its reserved capacity): 1 cell
 * in `stride`, cells with no tendency 1 in stride/keep_zero; NULL stops. */
int cress_set_tuple_sampling(cress_ctx* ctx, cress_mlp* m, int stride, float keep_zero, unsigned long long seed);

/* One HE-VI acoustic substep that allocates no device memory.  No
 * counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc from inside their time loop, such as a host model that keeps
 * all of its device arrays in a pool sized at start-up, or a framework
 * whose caching allocator owns the device.  No context is needed.
 *
 * The caller passes device buffers it owns: the old u, v, w, p' and the
 * four forcings (inputs) and the new u, v, w, p' (outputs), each in the
 * layout a(0:ni+1, 0:nj+1, 1:nk) with the x pitch padded to
 * round_up(ni+2, 32) floats, 16-byte aligned; base3d are host arrays as in
 * cress_set_base3d.  The small per-column data the kernel needs (base-state
 * columns, the w-system elimination factors, an error word) goes into one
 * fixed __device__ array of about 28 KB per GPU, resident until the process
 * exits; hence nk <= 256 (larger grids return CRESS_E_ARG).  A call
 * rewrites that array when its parameters (dims, spacing, dts, weicoe,
 * buyopt, base pointers, base centre columns) differ from the previous
 * call's on the device, and always clears its error word; calls whose
 * kernels overlap on the GPU race on it and must be serialized.  The
 * horizontal-uniformity scan of base3d runs only on such a change.  The
 * kernel is the context API's for cfg->tile (0-10; 11 is rejected).
 * The first call on a device looks up the
 * array's address with that device current; make it before any stream
 * capture begins.  The call is synchronous on `stream` (NULL = the default
 * stream) and returns CRESS_E_TIMEOUT if a bounded device-side wait gave up. */
int cress_hevi_substep_noalloc(const cress_cfg* cfg, float dts, const float* const* base3d,
                               const float* u_old, const float* v_old, const float* w_old,
                               const float* p_old, const float* ufrc, const float* vfrc,
                               const float* wfrc, const float* pfrc, float* u_new, float* v_new,
                               float* w_new, float* p_new, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CRESS_B200_H */
