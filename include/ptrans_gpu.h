/*
 * ptrans_gpu.h - C ABI of the B200 (sm_100a) Monte Carlo ray-tracing (RTMC)
 * phonon transport hot path.
 *
 * The reference solver (P-TRANS, Fortran module RTMC in src/RTMCphon.f90) runs
 *   RayTrace -> TransmissionFunction -> calcTransmit -> findCollisionSurface /
 *   calcSurfaceDistance* -> reflect* / determin* -> tally
 * and then effectiveMFP (Simpson over the incident angle) and the kappa sum of
 * fileoutput.  This header is the drop-in seam for that path: every entry point
 * uses only int32_t / int64_t / uint64_t / double, plain pointers and structs of
 * those, so a Fortran host binds it with ISO_C_BINDING (bind(C)).
 *
 * Conventions
 *  - Every function returns an int status: PTG_OK (0) on success, matching the
 *    reference loaders' "status /= 0 means error" convention
 *    (src/RTMCphon.f90:254-269).  RayTrace's inverted logical status
 *    (src/RTMCphon.f90:3427-3432) stays on the Fortran side.
 *  - Indices inside arrays follow the reference: materials and grains are
 *    1-based where the reference is 1-based (grain_to, material ids); array
 *    positions are 0-based.  Two-dimensional arrays are Fortran column-major.
 *  - Lengths are in nm, like the reference's box and mean free paths.
 *  - The caller owns every input and output array.  A handle owns device
 *    buffers only; no caller pointer is kept past a call.
 *  - A handle is not re-entrant: one handle per host thread, one CUDA stream
 *    per handle.
 *
 * Random numbers: counter-based Philox4x32-10.  Key = (lo32(seed), hi32(seed)),
 * counter = (flight_no, sub | stream<<8, lo32(sample), hi32(sample)) where
 *   sample = task * np + particle      (particle 0-based, 0 <= particle < np)
 *   flight_no = 0 for the emission draws, n >= 1 for the n-th free flight.
 * The task numbering is fixed by this header (see ptg_run), so a trajectory is
 * the same whichever rank, kernel or launch runs it.
 */
#ifndef PTRANS_GPU_H
#define PTRANS_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PTG_OK              0
#define PTG_ERR_INVALID     1  /* bad argument or inconsistent input        */
#define PTG_ERR_CUDA        2  /* a CUDA runtime call failed                 */
#define PTG_ERR_NO_DEVICE   3  /* no usable sm_100 device                    */
#define PTG_ERR_TIMEOUT     4  /* a bounded device wait gave up              */
#define PTG_ERR_LOST        5  /* lost-phonon fraction above the set limit   */
#define PTG_ERR_NOMEM       6  /* allocation failed                          */
#define PTG_ERR_IO          7  /* file missing or malformed                  */
#define PTG_ERR_UNSUPPORTED 8  /* combination not implemented                */

/* ---- enumerations (values equal the reference's parameters) ------------ */
/* src/RTMCphon.f90:72-74 */
#define PTG_SHAPE_POLYGON   1
#define PTG_SHAPE_SPHERE    2
#define PTG_SHAPE_CYLINDER  3   /* infinite cylinder, axis parallel to z */
/* extension: a right circular cylinder of finite length with flat end caps
   and any axis.  In ptg_geometry its surface record holds the two end
   points of the axis as a closed vertex list (nvertex = 2: A, B, A), the
   centre (A+B)/2 and the radius; in ptg_model the grain's generatrix is the
   centre and grain_axis the vector B - A. */
#define PTG_SHAPE_CAPPED    4
/* src/RTMCphon.f90:77-79 */
#define PTG_TRANS_VALUE     1
#define PTG_TRANS_GAMMA     2
#define PTG_TRANS_TBC       3
/* src/RTMCphon.f90:127-132 */
#define PTG_MFP_MATTHIESSEN 1   /* no MeanFreePath key: ballistic MC + Matthiessen */
#define PTG_MFP_GRID        2   /* MeanFreePath grid + linear interpolation        */
#define PTG_MFP_PER_MODE    3   /* extension: each mode run at its own bulk MFP    */
#define PTG_GRAIN_VORONOI   1
#define PTG_GRAIN_BRICKS    2
/* box face boundary kind (extension; 0 keeps the reference behaviour:
   x faces absorb, the other faces reflect with CellSpecularity) */
#define PTG_FACE_REFERENCE  0
#define PTG_FACE_PERIODIC   1
/* kernel selection */
#define PTG_PREC_FP32       0   /* persistent FP32 kernel, FP64 tallies       */
#define PTG_PREC_FP64       1   /* plain FP64 one-phonon-per-thread kernel    */

/* material_to codes in ptg_model.surf_material_to */
#define PTG_MATERIAL_INTERNAL  0   /* "Internal": connects to the fill grain */
#define PTG_MATERIAL_BOUNDARY (-1) /* "Boundary" or any name not in the list */

/*
 * Raw structure description: what loadMCP reads from a .mcp file
 * (loadParameterBox src/RTMCphon.f90:279-420, loadParameterTransmission
 * :749-890, loadGeometry :894-1251).  ptg_geometry_build turns it into the
 * built geometry exactly as setupBoxGrain / setupSurfaceGeometry /
 * setupSurfaceTransmissivity / setupFillGrain do (:1253-1491).
 */
typedef struct ptg_model {
  double box[3];            /* param%boxx/y/z = LXcell*NXcell ... [nm]          */
  double cellspec[6];       /* CellSpecularity for x-,x+,y-,y+,z-,z+            */
  int32_t face_kind[6];     /* PTG_FACE_* (extension); x faces must be 0        */
  double specfluc;          /* FluctuationSpecularity (Gaussian sigma)          */
  double scope[2];          /* ScopeY, ScopeZ                                   */
  double temperature;       /* temp [K]                                         */
  int32_t kind_grain;       /* PTG_GRAIN_VORONOI or PTG_GRAIN_BRICKS            */
  int32_t nmaterial;        /* Nm                                               */
  int32_t nt1, nt2;         /* "Nt" table shape                                 */
  const int32_t* tt_kind;   /* [(nt2+1)*nt1] param%kindTrans(nt2+1,nt1)         */
  const double* tt_trans;   /* [(nt2+1)*nt1] transmissivity, or gamma for      */
                            /*   Gamma/TBC (TBC already solved to gamma)       */
  const double* tt_spec;    /* [(nt2+1)*nt1] specularity                        */
  int32_t ngrain;           /* Ng                                               */
  const int32_t* grain_shape;       /* [ngrain] PTG_SHAPE_*                     */
  const double* grain_generatrix;   /* [3*ngrain]                               */
  const double* grain_diameter;     /* [ngrain] (sphere / cylinder)             */
  const int32_t* grain_material;    /* [ngrain] 1-based material index          */
  const int32_t* grain_nfacet;      /* [ngrain] facets (polygon grains), else 1 */
  const int32_t* facet_nvertex;     /* [nfacet_poly] vertices per facet         */
  const double* facet_vertex;       /* [3*sum(facet_nvertex)] open polygons     */
  const int32_t* surf_material_to;  /* [nsurf_model] PTG_MATERIAL_* or 1-based  */
  const int32_t* surf_grain_to;     /* [nsurf_model] grain_to as read           */
  const double* surf_spec;          /* [nsurf_model] or NULL: per-surface       */
                                    /*   specularity override (extension)       */
  uint64_t fluct_seed;              /* seed of the specularity fluctuation      */
  const double* grain_axis;         /* [3*ngrain] or NULL: axis vector B - A of */
                                    /*   PTG_SHAPE_CAPPED grains (extension)    */
} ptg_model;

/* Per-mode bulk phonon data as held in Anphon_type after loadAnphon
   (src/RTMCphon.f90:149-163, :661-733).  Arrays are (nbranch,nkpoint)
   column-major: element (ib,ik) is at ib + nbranch*ik. */
typedef struct ptg_spectrum {
  int32_t nbranch, nkpoint;
  double rtemp;             /* RTemp [K]                                        */
  double vol;               /* vol                                              */
  const double* omega;      /* rad/s (file value * 0.03 * 2*pi * 1e12)          */
  const double* tau;        /* ps, as read                                      */
  const double* vel;        /* m/s                                              */
  const double* mfp;        /* as read (unused by the transport)                */
  const double* weight;     /* k-point weight                                   */
} ptg_spectrum;

/*
 * Built geometry: the flattened form of vgrain(0:...) (src/RTMCphon.f90:94-124).
 * Grain 0 is the box (6 surfaces in the order x-,x+,y-,y+,z-,z+), grains
 * 1..ngrain the .mcp grains, and for bricks the fill grain ngrain+1.
 * Surfaces of grain g are [grain_begin[g], grain_begin[g+1]).
 */
typedef struct ptg_geometry {
  double box[3];
  double scope[2];
  int32_t face_kind[6];
  int32_t kind_grain;
  int32_t ngrain;           /* .mcp grains                                      */
  int32_t igrain_fill;      /* -1 (voronoi) or ngrain+1 (bricks)                */
  int32_t nmaterial;
  int32_t ngrain_total;     /* ngrain+1, plus 1 for the fill grain              */
  int32_t nsurf;            /* all surfaces of all grains                       */
  int32_t nvertex_total;    /* closed polygons: nvertex+1 entries per surface   */
  const int32_t* grain_begin;       /* [ngrain_total+1]                         */
  const int32_t* grain_incident;    /* [ngrain_total]                           */
  const double* grain_generatrix;   /* [3*ngrain_total]                         */
  const int32_t* shape;             /* [nsurf] PTG_SHAPE_*                      */
  const int32_t* nvertex;           /* [nsurf]                                  */
  const int32_t* vertex_begin;      /* [nsurf] offset (in vertices)             */
  const double* vertex;             /* [3*nvertex_total]                        */
  const double* normal;             /* [3*nsurf]                                */
  const double* tangent;            /* [9*nsurf] tangent(:,1..3) column-major   */
  const double* center;             /* [3*nsurf]                                */
  const double* radius;             /* [nsurf]                                  */
  const int32_t* kind_trans;        /* [nsurf] PTG_TRANS_*                      */
  const double* specularity;        /* [nsurf]                                  */
  const double* trans_param;        /* [nsurf] value (VALUE) or gamma           */
  const int32_t* grain_inside;      /* [nsurf]                                  */
  const int32_t* grain_outside;     /* [nsurf]                                  */
  const int32_t* internal;          /* [nsurf] 0/1                              */
  const int32_t* incident;          /* [nsurf] 0/1                              */
  const int32_t* material1;         /* [nsurf]                                  */
  const int32_t* material2;         /* [nsurf]                                  */
} ptg_geometry;

/* Handle options, fixed at ptg_create. Zero-initialise and set what you need. */
typedef struct ptg_options {
  int32_t device;           /* CUDA device ordinal                              */
  int32_t block_size;       /* persistent kernel threads per block (0 = tuned)  */
  int32_t blocks_per_sm;    /* persistent kernel residency (0 = occupancy)      */
  int32_t regen_threshold;  /* idle lanes before a warp refills (0 = 2)         */
  int32_t ref_quirks;       /* 1: a lost phonon also counts as transmitted      */
                            /*    (src/RTMCphon.f90:1701 then :1833)            */
  int32_t bvh_leaf;         /* BVH leaf size (0 = tuned, < 0 = no BVH): grains  */
                            /* with more than 32 candidate surfaces get a BVH   */
  int64_t max_flights;      /* per-trajectory cap, lost when reached (0 = 1e7)  */
  double lost_limit;        /* PTG_ERR_LOST if lost/total exceeds it (0 = off)  */
  int64_t chunk;            /* samples per work-queue chunk (0 = tuned)         */
  int32_t tune_flags;       /* persistent kernel variants (autotuner):          */
                            /*   bit 0: no safe-distance p-p fast path          */
                            /*   bit 1: no tail phase (one lane per phonon to   */
                            /*          the end)                                */
                            /*   bit 2: test only: the shared-memory staging    */
                            /*          copy is not issued, so its bounded wait */
                            /*          runs out and the call returns           */
                            /*          PTG_ERR_TIMEOUT                         */
  int32_t fast_steps;       /* fast p-p flights per iteration before a warp     */
                            /* goes on only while half its lanes still can      */
                            /* (at most 4x; 0 = 4 for structures without BVH or */
                            /* capped cylinders, 20 for the others, 8 in a      */
                            /* batched launch)                                  */
  int32_t coop_lanes;       /* once the work queue is dry, a warp with at most  */
                            /* this many live phonons hands them over to the    */
                            /* tail phase, a second kernel that gives           */
                            /* each a warp of 32 cooperating lanes (0 = 32)     */
  int32_t reserved;         /* reserved, must be 0                              */
} ptg_options;

/*
 * One transport run.  Tasks are numbered
 *   MATTHIESSEN / PER_MODE : task = ib + nb*(ik + nk*ia)
 *   GRID                   : task = ib + nb*(ik + nk*(s + nmfp*ia))
 * with ia in [0, nangle-2] (the last angle, pi/2, is never simulated,
 * src/RTMCphon.f90:1576) and theta_ia = ia/(nangle-1) * pi/2
 * (src/RTMCphon.f90:1554-1556).  Rank r of nranks runs the particles
 * p = r, r+nranks, ... of every task (src/RTMCphon.f90:1627).
 */
typedef struct ptg_run {
  int32_t kind_mfp;         /* PTG_MFP_*                                        */
  int32_t nangle;           /* odd, >= 3 (Simpson)                              */
  int64_t np;               /* particles per task                               */
  int32_t nmfp;             /* GRID: number of grid points                      */
  const double* mfp_grid_nm;/* GRID: [nmfp] ascending, > 0                      */
  uint64_t seed;
  int32_t stream;           /* 0..2^24-1, separates runs that share a seed      */
  int32_t rank, nranks;     /* particle striding (nranks >= 1)                  */
  int32_t precision;        /* PTG_PREC_FP32 or PTG_PREC_FP64                   */
  double temperature;       /* param%temperature [K] (tau rescale, heat capacity) */
  int32_t nbins;            /* per-frequency-bin outputs (0 = none)             */
  double bin_omega_min, bin_omega_max;   /* rad/s                               */
  double scatter_scale;     /* s: intrinsic rates times s, i.e. every mode's    */
                            /* bulk MFP divided by s (0 = 1); grid MFPs are    */
                            /* sampling points and do not change               */
} ptg_run;

/* Results of ptg_kappa.  Pointers are caller-owned outputs (NULL = skip). */
typedef struct ptg_kappa_out {
  double kappa;             /* W m^-1 K^-1, sum of Thermal_conductivity         */
  double kappa_stderr;
  double* bin_T;            /* [nbins] flux-weighted <T> per frequency bin      */
  double* bin_T_stderr;     /* [nbins]                                          */
  double* emfp_nm;          /* [nbranch*nkpoint] effective MFP per mode [nm]    */
  double* transmit;         /* [ntask_total + angle padding] see ptg_transmission */
  uint64_t* counts;         /* [ntask] transmitted counts of this rank          */
  uint64_t flights;         /* free flights simulated by this call              */
  uint64_t lost;            /* lost phonons                                     */
  uint64_t samples;         /* trajectories simulated                           */
  double kernel_ms;         /* device time of the transport kernel(s)           */
} ptg_kappa_out;

/* Statistics of the last call on a handle. */
typedef struct ptg_stats {
  uint64_t flights, lost, samples, capped;
  double kernel_ms;         /* CUDA-event time of the transport kernel          */
  double reduce_ms;         /* CUDA-event time of the kappa reduction kernel    */
  int32_t launches;         /* kernels launched by the call                     */
  int32_t grid, block;      /* transport launch shape                           */
  uint64_t h2d_bytes;       /* host-to-device bytes copied by the call          */
  uint64_t d2h_bytes;       /* device-to-host bytes copied by the call          */
  uint64_t max_traj_flights;/* longest trajectory (free flights), FP32 kernel   */
  double drain_ms;          /* FP32 kernel: start until the work queue ran dry  */
  double tail_ms;           /* FP32 kernel: queue dry until the last warp ended */
  uint64_t full_flights;    /* FP32 kernel: flights taken with the full test     */
  uint64_t safe_balls;      /* FP32 kernel: safe balls computed                 */
  uint64_t coop_rounds;     /* FP32 kernel: warp-cooperative rounds             */
  uint64_t coop_flights;    /* FP32 kernel: p-p flights taken in those rounds   */
  uint64_t box_tests;       /* FP32 kernel: BVH node boxes tested (32-bit lane  */
                            /*   counters: exact below 2^32 tests per thread)   */
  uint64_t surface_tests;   /* FP32 kernel: grain surfaces tested (box faces    */
                            /*   are one slab test and not counted)             */
  double drain_kernel_ms;   /* FP32: CUDA-event time of the drain-phase kernel  */
  double tail_kernel_ms;    /* FP32: CUDA-event time of the tail phase (its
                               ordering kernel and the tail-phase kernel)      */
                            /*   (0 when the tail phase is off)                 */
  uint64_t tail_phonons;    /* FP32: phonons the drain phase handed over        */
  uint64_t tail_flights;    /* FP32: free flights taken in the tail phase       */
  uint64_t tail_refused;    /* FP32: hand-overs refused because the tail list   */
                            /*   was full (those phonons stayed in the drain)   */
} ptg_stats;

typedef struct ptg_handle ptg_handle;
typedef struct ptg_geombuf ptg_geombuf;

/* ---- host-side geometry construction (no device needed) ---------------- */

/* Builds the geometry as loadGeometry/setupBoxGrain/setupFillGrain do.
   Replaces src/RTMCphon.f90:894-1491 (the part after the text parse). */
int ptg_geometry_build(const ptg_model* model, const ptg_spectrum* spec,
                       ptg_geombuf** out);
const ptg_geometry* ptg_geombuf_view(const ptg_geombuf* buf);
void ptg_geombuf_free(ptg_geombuf* buf);

/* Parses a .mcp file (src/RTMCphon.f90:252-1251).  The returned buffer owns
   the ptg_model arrays; anphon_name receives the first material name
   (the reference loads Materials/<name>.anphon, :671). */
typedef struct ptg_mcpbuf ptg_mcpbuf;
int ptg_mcp_load(const char* path, ptg_mcpbuf** out);
const ptg_model* ptg_mcpbuf_model(const ptg_mcpbuf* buf);
int ptg_mcpbuf_info(const ptg_mcpbuf* buf, int64_t* np, int32_t* nangle,
                    int32_t* kind_mfp, int32_t* nmfp, double* mfp_grid_nm,
                    int32_t* particle_trace, char* material1, int32_t len);
void ptg_mcpbuf_free(ptg_mcpbuf* buf);

/* Reads / writes the .anphon mode table (src/RTMCphon.f90:661-733). */
typedef struct ptg_anphonbuf ptg_anphonbuf;
int ptg_anphon_load(const char* path, ptg_anphonbuf** out);
const ptg_spectrum* ptg_anphonbuf_spectrum(const ptg_anphonbuf* buf);
void ptg_anphonbuf_free(ptg_anphonbuf* buf);
int ptg_anphon_write(const char* path, const ptg_spectrum* s);

/* ---- device handle ------------------------------------------------------ */

/* Uploads geometry and spectrum to the device and sizes the work buffers. */
int ptg_create(const ptg_geometry* geom, const ptg_spectrum* spec,
               const ptg_options* opt, ptg_handle** out);
/* Replaces the spectrum (same nbranch, nkpoint). */
int ptg_set_spectrum(ptg_handle* h, const ptg_spectrum* spec);
void ptg_destroy(ptg_handle* h);
const char* ptg_strerror(int status);

/*
 * The body of TransmissionFunction (src/RTMCphon.f90:1544-1604) for one gray
 * mean free path: fills transmit(nbranch,nkpoint,nangle) column-major with
 * (transmitted particles of this rank)/np, transmit(:,:,nangle) = 0, exactly
 * what calcTransmit leaves before the MPI_Allreduce (:1584-1590).
 * mfp_nm = 1e10 means ballistic (:1686-1690).  stderr_opt (same shape, may be
 * NULL) receives sqrt(T(1-T)/np) with T the rank-local value.
 * precision selects the kernel (PTG_PREC_FP32 / PTG_PREC_FP64).
 */
int ptg_transmission(ptg_handle* h, double mfp_nm, int32_t nangle, int64_t np,
                     int32_t rank, int32_t nranks, uint64_t seed,
                     int32_t precision, double* transmit, double* stderr_opt);

/*
 * Transport for every task of a run, then effectiveMFP (Simpson,
 * src/RTMCphon.f90:2418-2451) and the kappa sum of fileoutput
 * (:2645-2755) as an FP64 reduction on the device.  out->transmit, when set,
 * has nb*nk*nmfp_eff*nangle entries laid out like the task numbering with
 * the angle slowest (nmfp_eff = nmfp for GRID, else 1).
 */
int ptg_kappa(ptg_handle* h, const ptg_run* run, ptg_kappa_out* out);

/*
 * Host FP64 assembly of kappa from (all-reduced) transmitted counts, for a
 * multi-rank caller that sums ptg_kappa_out.counts across ranks first, as the
 * reference sums transmit with MPI_Allreduce (src/RTMCphon.f90:1587).
 * counts has one entry per task (ptg_run numbering, angle nangle-1 excluded).
 */
int ptg_kappa_from_counts(const ptg_geometry* geom, const ptg_spectrum* spec,
                          const ptg_run* run, const uint64_t* counts,
                          ptg_kappa_out* out);

/*
 * The reference's result files from the counts of a run: replaces fileoutput
 * (src/RTMCphon.f90:2601-2881), called after RayTrace's MFP loop with
 * SEMFP from effectiveMFP (:2418-2451).  Writes thermalproperty.out,
 * effectiveMFP.out and phononconductivity.out in the directory of geofile
 * (the .mcp path, as the reference derives it, :2629-2632), with the
 * reference's record layouts and Fortran edit descriptors; only
 * thermalproperty.out when geom->nmaterial > 1, as the reference.
 * Returns PTG_ERR_IO when a file cannot be written.
 */
int ptg_write_outputs(const char* geofile, const ptg_geometry* geom, const ptg_spectrum* spec,
                      const ptg_run* run, const uint64_t* counts);
/*
 * Interface parameter of a "TBC" transmission entry: GammaDeterm
 * (src/RTMCphon.f90:2499-2599, called from the .mcp reader at :856-873).
 * Newton's method for the gamma whose transmissivity
 * T = 1/(gamma omega/omega_max + 1) over the modes of `material` gives the
 * boundary conductance tbc [W m^-2 K^-1] (the .mcp value times 1e6, as
 * ptg_mcp_load stores it in tt_trans); the result goes into tt_trans in
 * place of the conductance.  PTG_ERR_INVALID when gamma < 0 ("Gamma cannot
 * determine").
 */
int ptg_gamma_from_tbc(const ptg_spectrum* material, double temperature, double tbc,
                       double* gamma);
/* The writer's rendering of one Fortran edit descriptor (kind 0: Iw,
   1: Fw.d with w = 0 for F0.d, 2: Ew.d) into out (cap bytes, NUL ended). */
int ptg_fortran_format(int32_t kind, double v, int32_t w, int32_t d, char* out, int32_t cap);

/*
 * Adjoint (path-reweighting) derivatives of kappa.  A forward pass of the
 * persistent FP32 kernel records which samples leave through x+; a second
 * pass re-generates exactly those trajectories from their Philox counters
 * (no path is stored) and accumulates, with the weight dkappa/dT_task / np,
 *   d log P / d p_k = sum over events on surface record k of 1/p_k for a
 *                     specular choice and -1/(1-p_k) for a diffuse one,
 *   d log P / d s   = (intrinsic events) - (path length) / lambda
 * for the scale s of the intrinsic rates (PER_MODE; MATTHIESSEN and GRID add
 * the analytic term of the bulk-MFP dependence of their kappa rule).
 * Derivatives are per surface record of the built geometry; records with
 * p = 0 or 1 get NaN (the estimator is biased at the end points).  Standard
 * errors come from 8 interleaved sample batches.  The listing pass keeps
 * 8 bytes per sample of the run on the device (at most 2^31 samples per
 * call, PTG_ERR_UNSUPPORTED beyond).
 */
typedef struct ptg_adjoint_out {
  double kappa, kappa_stderr;
  double* dk_dp;            /* [nsurf] dkappa / d specularity of each record     */
  double* dk_dp_stderr;     /* [nsurf]                                           */
  double dk_dscale, dk_dscale_stderr;
  uint64_t flights;         /* forward + replay free flights                     */
  uint64_t replayed;        /* transmitted samples re-generated                  */
  uint64_t mismatched;      /* replays that did not transmit again (expect 0)    */
  double kernel_ms;         /* forward + replay transport time                   */
} ptg_adjoint_out;
int ptg_adjoint(ptg_handle* h, const ptg_run* run, ptg_adjoint_out* out);

/*
 * Batched screening: many structures (each a built geometry with its own
 * particle count, seed and stream) share one spectrum and run settings and
 * run in ONE persistent kernel launch, replayed as a CUDA graph by
 * ptg_batch_run.  Each geometry gets exactly the counts of its own ptg_kappa
 * run with the same np, seed and stream (the FP32 kernel), i.e. the
 * reference's RayTrace repeated per structure (src/RTMCphon.f90:3334-3433).
 * The run's np, seed and stream are ignored (per item instead); the tables
 * are built once, so a batch object is re-run without any host work.
 */
typedef struct ptg_batch ptg_batch;
typedef struct ptg_batch_item {
  const ptg_geometry* geom;
  int64_t np;               /* particles per (mode, angle) task              */
  uint64_t seed;
  int32_t stream;
} ptg_batch_item;
typedef struct ptg_batch_out {
  double* kappa;            /* [nitems]                                      */
  double* kappa_stderr;     /* [nitems]                                      */
  double* bin_T;            /* [nitems*nbins]                                */
  double* bin_T_stderr;     /* [nitems*nbins]                                */
  uint64_t* counts;         /* [nitems*ntask] or NULL                        */
  uint64_t flights, lost, samples;
  double graph_ms;          /* device time of the graph launch               */
} ptg_batch_out;
int ptg_batch_create(const ptg_batch_item* items, int32_t nitems, const ptg_spectrum* spec,
                     const ptg_run* run, const ptg_options* opt, ptg_batch** out);
int ptg_batch_run(ptg_batch* b, ptg_batch_out* out);
/*
 * Per-geometry adjoint of a batch (no counterpart in the reference): what
 * ptg_adjoint gives for each geometry's own run, from two batched launches
 * over all geometries - a forward pass that lists the samples leaving
 * through x+ as (global task, particle) ids, then, after the host has
 * assembled every geometry's kappa and d kappa / d T_task, one replay of
 * all listed samples from their Philox counters that accumulates each
 * sample's score into its geometry's slice.  dk_dp and dk_dp_stderr hold
 * the geometries' surface records one after the other (geometry g starts at
 * the sum of the earlier geometries' nsurf); NaN where p is 0 or 1.
 */
typedef struct ptg_batch_adjoint_out {
  double* kappa;            /* [nitems]                                      */
  double* kappa_stderr;     /* [nitems]                                      */
  double* dk_dp;            /* [sum of nsurf]                                */
  double* dk_dp_stderr;     /* [sum of nsurf]                                */
  double* dk_dscale;        /* [nitems]                                      */
  double* dk_dscale_stderr; /* [nitems]                                      */
  uint64_t flights;         /* forward + replay free flights                 */
  uint64_t replayed;        /* transmitted samples re-generated              */
  uint64_t mismatched;      /* replays that did not transmit again (0)       */
  double kernel_ms;         /* device time of the two launches               */
} ptg_batch_adjoint_out;
int ptg_batch_adjoint(ptg_batch* b, ptg_batch_adjoint_out* out);
void ptg_batch_destroy(ptg_batch* b);

/*
 * Bounds-checked build (no counterpart in the reference, whose debug aids
 * are its verbose self-checks, src/RTMCphon.f90:1695-1703, 1711-1731):
 * libptrans_b200_check.so, the same library built with -DPT_CHECK, checks
 * every geometry-blob index the FP32 kernels read (surfaces, edges,
 * candidates, BVH nodes) and that every live phonon's state is finite; a
 * failed check is counted, its access redirected to a valid element, and
 * the kernel goes on (it never traps).  ptg_check_report returns, for a
 * device, the number of failed checks since the last reset, the code of the
 * first (1 index out of range, 2 non-finite state) and its index (the blob
 * unit, or the task); reset != 0 clears them.  Regular builds return
 * PTG_ERR_UNSUPPORTED.
 */
int ptg_check_report(int32_t device, int64_t* violations, int32_t* first_code, int32_t* first_index,
                     int32_t reset);

/*
 * Test hook (no counterpart in the reference): the next `after` allocations
 * the library makes succeed and every later one fails - device buffers are
 * not requested from CUDA and host objects are not created - so that every
 * entry point's out-of-memory path can be exercised; the calls return
 * PTG_ERR_NOMEM and leave their handles usable.  after < 0 turns it off.
 */
int ptg_debug_fail_allocations(int64_t after);

/* Statistics of the last transport call on h. */
int ptg_last_stats(const ptg_handle* h, ptg_stats* st);

/*
 * Trajectory trace by replay: replaces the trace.out output of calcTransmit
 * (src/RTMCphon.f90:1661-1665, 1818-1831, file set-up :3373-3383), which
 * the reference writes from inside its hot loop.  Here the transport
 * kernels write nothing per flight; ptg_trace re-generates the FP32
 * trajectories of the listed samples (global sample ids task * np + p of
 * the run's numbering) from their Philox counters, one lane per sample with
 * the full intersection test on every flight (the same trajectory as any
 * other path of the kernel), and returns per sample the number of
 * positions npos (emission point + one per free flight), the exit side
 * (0 lost, 1 x-, 2 x+) and, when pos is not NULL, the positions
 * (3 floats each, sample i at the running sum of the earlier npos); a
 * buffer smaller than the sum of npos gives PTG_ERR_INVALID with npos and
 * end_side filled.  ptg_write_trace picks particle_trace samples every
 * interval_trace = ntask * np / particle_trace ids (the reference's
 * interval, one rank) and writes the reference's trace.out: its header,
 * one record per position (x y z as FP32 values, 9 significant digits),
 * two blank records after each phonon.
 */
int ptg_trace(ptg_handle* h, const ptg_run* run, int64_t n, const uint64_t* samples,
              int64_t cap_positions, float* pos, int64_t* npos, int32_t* end_side);
int ptg_write_trace(ptg_handle* h, const ptg_run* run, int32_t particle_trace, const char* path);

/*
 * Options of a live handle and the autotuner - no counterpart in the
 * reference, whose OpenMP loop has a fixed static schedule
 * (src/RTMCphon.f90:1573).
 *
 * ptg_set_options replaces the handle's options (same device); a new
 * bvh_leaf rebuilds the device geometry.  ptg_autotune times ptg_kappa with
 * `run` in FP32 (best of `reps` calls per trial) while it varies, one at a
 * time, bvh_leaf (when a grain has a BVH), block_size, blocks_per_sm,
 * coop_lanes, fast_steps, regen_threshold and chunk; it leaves the fastest
 * options on the handle and in *best, with their kernel time in *best_ms.
 * Trajectories depend only on their Philox counters, so no option changes a
 * result.  The call runs about 20 trials of the given run: tune on a run
 * with fewer particles when the full one is long.
 */
int ptg_get_options(const ptg_handle* h, ptg_options* out);
int ptg_set_options(ptg_handle* h, const ptg_options* opt);
int ptg_autotune(ptg_handle* h, const ptg_run* run, int32_t reps, ptg_options* best,
                 double* best_ms);

/*
 * ptg_transmission_noalloc - no counterpart in the reference; an addition for
 * hosts that cannot allocate memory while they run (device memory reserved up
 * front by another framework, or a service that must keep a fixed
 * footprint).  It computes what ptg_transmission computes with
 * PTG_PREC_FP32 (same counts, so the same transmit array; the same
 * lost-phonon limit; the same ptg_last_stats record, kernel times aside) but
 * allocates no device or host memory: the kernels' scratch (work-queue
 * counter, statistics, tallies, task and chunk tables, a 65536-phonon
 * tail-phase list and its order; hand-overs past its capacity stay in the
 * drain phase and are counted in ptg_stats.tail_refused) lives in one static
 * device array of fixed size (about 9.3 MB) that every GPU loading the
 * library keeps until
 * exit, and the caller's transmit array receives the counts before they are
 * divided by np in place (on PTG_ERR_TIMEOUT or PTG_ERR_CUDA after the
 * launch it is zeroed).  Limits: nbranch*nkpoint*(nangle-1) <=
 * PTG_NOALLOC_MAX_TASKS, nangle <= 64; larger runs return PTG_ERR_INVALID.
 * The first call on a device looks up the array's address (make it before
 * any stream capture).  All calls share the array: calls whose GPU work
 * overlaps race and must be serialised by the caller.
 */
#define PTG_NOALLOC_MAX_TASKS  16384
#define PTG_NOALLOC_MAX_CHUNKS 65536
int ptg_transmission_noalloc(ptg_handle* h, double mfp_nm, int32_t nangle, int64_t np,
                             int32_t rank, int32_t nranks, uint64_t seed, double* transmit);

/* Debug / replay: runs the FP64 kernel for one task and writes, per particle,
   the exit side (0 lost, 1 x-, 2 x+) and the number of free flights. */
int ptg_replay_task(ptg_handle* h, const ptg_run* run, int64_t task,
                    int32_t* end_side, uint32_t* flights, double* final_pos);

#ifdef __cplusplus
}
#endif
#endif /* PTRANS_GPU_H */
