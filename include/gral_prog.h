/*
 * gral_prog.h -- C ABI of the B200 prognostic microscale flow solver.
 *
 * Drop-in for GRAL's `PrognosticFlowfield.Calculate()` (PrognosticFlowfield.cs:32),
 * which MicroscaleFlat.Calculate (MicroscaleFlat.cs:381) and MicroscaleTerrain.Calculate
 * (MicroscaleTerrain.cs:847) call once per weather situation.  The reference method takes no
 * arguments and works on `Program.*` statics; this ABI passes the same data explicitly:
 *
 *   gral_params  -- the scalars the reference reads from Program.* and from the control files
 *                   (turbulence_model.txt, Integrationtime.txt, relaxation_factors.txt,
 *                   building_roughness.txt, in.dat flags), PrognosticFlowfield.cs:147-291.
 *   gral_static  -- per-grid arrays that do not change during a solve (KKART, ADVDOM, CUTK, COV,
 *                   VEG, DZK, HOKART, roughness), ProgramDeclarations.cs:84-92, 456-484.
 *   gral_fields  -- the wind (and k-eps) fields read and written by the solve: UK, VK, WK,
 *                   TURB, TDISS, ProgramDeclarations.cs:432-440, 464-468.
 *
 * Host layout of every 3-D array: [NII+2][NJJ+2][NKK+2] float, k fastest, indices as in the
 * reference (1-based i, j, k; UK on west faces, VK on south faces, WK on bottom faces), so a
 * jagged `float[][][]` row of the reference maps to one contiguous run of NKK+2 floats.
 * 2-D per-column arrays are [NII+2][NJJ+2], j fastest.
 *
 * All functions return GRAL_OK (0) or a negative GRAL_E* code; nothing aborts or throws across
 * the ABI.  A context is used by one host thread at a time; calls are synchronous.  Signatures
 * hold only pointers, integers, floats and POD structs (blittable for P/Invoke under
 * DisableRuntimeMarshalling, GRAL.csproj:23).
 */
#ifndef GRAL_PROG_H
#define GRAL_PROG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRAL_PROG_ABI_VERSION 1

#define GRAL_OK 0
#define GRAL_EINVAL (-1)     /* bad dimensions, pointers or parameters */
#define GRAL_ENOMEM (-2)     /* device or host allocation failed / batch exceeds capacity */
#define GRAL_ECUDA (-3)      /* CUDA runtime error (text via gral_prog_last_error) */
#define GRAL_ETIMEDOUT (-4)  /* a bounded device-side wait gave up */
#define GRAL_ENONFINITE (-5) /* non-finite value in the solved fields */
#define GRAL_ENODEV (-6)     /* no usable CUDA device */
#define GRAL_ESTATE (-7)     /* call out of order (e.g. store before load) */
#define GRAL_ETOOLARGE (-8)  /* grid larger than a fixed-size entry point accepts */

/* Solver scalars.  Defaults in brackets are the reference defaults. */
typedef struct gral_params {
    int32_t nii, njj, nkk;        /* Program.NII/NJJ/NKK */
    int32_t kadvmax;              /* Program.KADVMAX (MicroscaleFlat.cs:196) */
    int32_t vert_cells_ff;        /* Program.VertCellsFF (micro_vert_layers.txt) */
    float dxk, dyk;               /* Program.DXK/DYK */
    int32_t turbulence_model;     /* 0 no diffusion, 1 mixing length [1], 2 k-eps */
    int32_t simd_width;           /* model-1 parity width: 8 = Vector<float> path [8], 16 = the
                                     Vector512 routines (Program.UseVector512Class) */
    int32_t iteration_steps_min;  /* [100] Integrationtime.txt line 1 */
    int32_t iteration_steps_max;  /* [500] Integrationtime.txt line 2 */
    int32_t conv_cadence;         /* [100] convergence test every this many iterations */
    double conv_threshold;        /* [0.012] DeltaMean / topwind^2 threshold */
    float relax, relaxp;          /* [0.1, 1] relaxation_factors.txt */
    float building_z0;            /* [0.001] building_roughness.txt */
    float coriolis;               /* Program.CorolisParam */
    float potdtdz;                /* Program.PotdTdz (k-eps buoyancy) */
    int32_t ref_i, ref_j;         /* Program.SubDomainRefPos */
    int32_t quantise;             /* [1] Frund rounding as the reference; 0 switches it off */
    int32_t turb_init;            /* model != 1: 0 = initialise TURB/TDISS as the reference's
                                     default meteo branch (PrognosticFlowfield.cs:410-510);
                                     1 = take TURB/TDISS from gral_fields as given */
    float std_dev_v, std_dev_w;   /* Program.StdDeviationV/W [1, 1] */
    float bd_lay_height;          /* Program.BdLayHeight */
    float v0_1;                   /* Program.V0[1] (sigma_v used by the TURB initialisation) */
    int32_t post_diagnostic;      /* [0] 1: after the prognostic solve, run what the flat-terrain
                                     caller runs next on the same fields: DiagnosticFlowfield.
                                     Calculate (10 pressure iterations over the full height,
                                     DiagnosticFlowfield.cs:24-436) and the final vertical
                                     velocity of the columns outside the prognostic sub-domains
                                     (MicroscaleFlat.cs:389-462) */
} gral_params;

/* Per-grid inputs; shared by all situations of a batch. */
typedef struct gral_static {
    const int16_t *kkart;     /* Program.KKART   [NII+2][NJJ+2] */
    const uint8_t *advdom;    /* Program.ADVDOM  [NII+2][NJJ+2] (prognostic sub-domain mask) */
    const float *cutk;        /* Program.CUTK    [NII+2][NJJ+2] (building height above ground) */
    const float *cov;         /* Program.COV     [NII+2][NJJ+2] (vegetation cover) */
    const float *z0;          /* roughness the momentum/TKE wall laws look up per column
                                 (Z0Gramm[IUstern][JUstern] or Z0Gral[i][j]) [NII+2][NJJ+2] */
    const float *z0_init;     /* roughness of the TURB initialisation per column (model != 1) */
    const float *ob_init;     /* Obukhov length of the TURB initialisation per column */
    const float *ust_init;    /* friction velocity of the TURB initialisation per column */
    const float *veg;         /* Program.VEG [NII+2][NJJ+2][NKK+2], or NULL */
    const uint8_t *veg_mask;  /* 1 where Program.VEG[i][j] is not null; NULL = no vegetation */
    const float *dzk;         /* Program.DZK    [NKK+2] */
    const float *hokart;      /* Program.HOKART [NKK+2] */
} gral_static;

/* Per-situation fields, read and written in place. */
typedef struct gral_fields {
    float *uk, *vk, *wk;      /* [NII+2][NJJ+2][NKK+2] */
    float *turb, *tdiss;      /* same layout; required when turbulence_model != 1, else NULL */
} gral_fields;

#define GRAL_MAX_HISTORY 64

typedef struct gral_stats {
    int32_t iterations;          /* SIMPLE iterations executed */
    int32_t iteration_loops;     /* value of IterationLoops printed by the reference at exit */
    int32_t converged;           /* 1 if the cadence test stopped the loop */
    int32_t convergence_problem; /* DeltaFinish > DeltaFirst (PrognosticFlowfield.cs:1187) */
    double delta_first, delta_finish;
    int32_t n_history;
    double delta_history[GRAL_MAX_HISTORY];   /* _delta at each cadence test */
    int32_t uk_unrealistic, vk_unrealistic, wk_unrealistic;  /* PrognosticFlowfield.cs:1193 */
    double geschw_max;           /* GESCHW_MAX */
    float topwind, dtime;
    double frund;
    float last_delta_umax;
    float *trace_delta_umax;     /* optional, caller-owned: DeltaUMax per iteration */
    int32_t trace_capacity;
    double ms_total, ms_upload, ms_iterate, ms_download;
    int32_t layout;              /* device layout used: 0 slab (one warp per column), 1 interleaved
                                    (32 situations per group, one block per group-column) */
    int32_t launch_variant;      /* launch variant the autotuner kept: interleaved layout, the batched
                                    kernels' variant; slab layout, the schedule of the model-1 sweeps
                                    (0 diagonal-claim wavefront, 1+v strip variant v, 5 fused strips; GRAL_PROG_PLAIN_MODE
                                    forces one) */
    int32_t launches_per_iteration; /* kernel launches of one SIMPLE iteration in the kept configuration */
} gral_stats;

typedef struct gral_ctx gral_ctx;

/* Library version (GRAL_PROG_ABI_VERSION). */
int gral_prog_version(void);

/* Create a context for grids up to nii x njj x nkk and up to max_batch situations solved
 * together.  Replaces the reference's lazy allocation of UKS/VKS/WKS/DPMNEW
 * (PrognosticFlowfield.cs:45-103). */
int gral_prog_create(int32_t nii, int32_t njj, int32_t nkk, int32_t kadvmax,
                     int32_t max_batch, gral_ctx **out);

/* One situation: PrognosticFlowfield.Calculate() (PrognosticFlowfield.cs:32-1245).  Reads
 * `fields`, runs the SIMPLE loop to convergence or iteration_steps_max, writes the fields back.
 * `stats` may be NULL. */
int gral_prog_solve(gral_ctx *ctx, const gral_params *p, const gral_static *s,
                    gral_fields *f, gral_stats *stats);

/* n situations on the same grid, each with its own params and fields, solved together with a
 * per-situation convergence mask.  p, f and stats are arrays of length n (stats may be NULL). */
int gral_prog_solve_batch(gral_ctx *ctx, int32_t n, const gral_params *p, const gral_static *s,
                          gral_fields *f, gral_stats *stats);

/* A batch of n situations on one grid (as gral_prog_solve_batch) spread over ndev devices of this
 * node: devices[d] (a CUDA device ordinal; one may repeat) takes the contiguous shard of situations
 * [d*n/ndev, (d+1)*n/ndev) in a context of its own, created and released inside the call, each
 * shard solved by its own host thread with no exchange between devices (weather situations are
 * independent, Program.cs:403-742).  Results are those of n single solves.  Returns GRAL_OK, or
 * the code of the first shard in device order that failed; GRAL_EINVAL for ndev < 1, n < ndev or an
 * ordinal outside 0..cudaGetDeviceCount()-1.  stats may be NULL. */
int gral_prog_solve_batch_devices(int32_t ndev, const int32_t *devices, int32_t n, const gral_params *p,
                                  const gral_static *s, gral_fields *f, gral_stats *stats);

/* Independent situations whose grids differ (one gral_params, gral_static and gral_fields per
 * instance; GRAL solves such sets one after the other), several at once, each exactly as
 * gral_prog_solve does (results are identical to n single calls).  The instances are ordered by
 * device footprint, largest first; K slots (each a context, stream and host thread) take the K
 * largest, whose loads run one after the other, then every slot solves its instance and takes the
 * next largest one left as soon as it is done, reusing its buffers.  K is max_concurrent, further
 * limited to the largest instances whose footprints fit in hbm_bytes of device memory together
 * (0: 90 % of the free memory at the call; the largest instance is loaded first and its measured
 * footprint scales the others' by their field sizes).  status[b] receives
 * instance b's return code (the error text of a failed instance is not kept); the call returns
 * GRAL_OK when every instance succeeded, else the code of the first failed instance in index
 * order.  stats may be NULL. */
int gral_prog_solve_instances(int32_t n, const gral_params *p, const gral_static *s, gral_fields *f,
                              gral_stats *stats, int32_t *status, int32_t max_concurrent, uint64_t hbm_bytes);

/* Split form of gral_prog_solve_batch for callers that keep fields resident on the device:
 * load copies inputs to HBM and runs the set-up, iterate runs the SIMPLE loop on the loaded
 * situations, store copies results back.  solve_batch = load + iterate + store. */
int gral_prog_load(gral_ctx *ctx, int32_t n, const gral_params *p, const gral_static *s,
                   gral_fields *f);
int gral_prog_iterate(gral_ctx *ctx);
int gral_prog_store(gral_ctx *ctx, gral_fields *f, gral_stats *stats);

/* Phases of one SIMPLE iteration, in launch order, as reported by gral_prog_iterate_timed. */
#define GRAL_NUM_PHASES 10
#define GRAL_PHASE_BC 0          /* lateral and top boundary conditions, PrognosticFlowfield.cs:595-714 */
#define GRAL_PHASE_PRESSURE 1    /* divergence + pressure-correction TDMA sweep, :723-901 */
#define GRAL_PHASE_VELCORR 2     /* velocity correction with Frund rounding, :904-949 */
#define GRAL_PHASE_AVERAGE 3     /* staggered-grid averages, :958-1039 */
#define GRAL_PHASE_U 4           /* U momentum (U-prognostic-microscale_*.cs) */
#define GRAL_PHASE_V 5           /* V momentum */
#define GRAL_PHASE_W 6           /* W momentum */
#define GRAL_PHASE_TKE 7         /* k and eps transport (model 2) */
#define GRAL_PHASE_BOOKKEEPING 8 /* convergence bookkeeping, :1144-1178 */
#define GRAL_PHASE_FUSED 9       /* pressure, velocity correction, averages and U in one wavefront
                                    launch (slab layout, model 1); phases 1-4 then read 0 */

/* Instrumentation: runs exactly `iterations` SIMPLE iterations on the loaded situations (the
 * convergence bookkeeping still runs, so a situation that meets the reference's stop rule stops
 * updating), launching each phase separately with CUDA events between phases and no host
 * synchronisation inside the run.  phase_ms[GRAL_NUM_PHASES] receives the summed device time of
 * each phase, total_ms the device time of the whole run.  Either pointer may be NULL. */
int gral_prog_iterate_timed(gral_ctx *ctx, int32_t iterations, double *phase_ms, double *total_ms);

/* GRAL flow-field and turbulence cache files (GFFWrite.cs, GFFRead.cs).  The reference writes
 * each as a zip archive holding one entry; these calls produce and consume that entry's bytes
 * (the host does the zip step).  Every payload starts with the same 32-byte little-endian header:
 * int32 NKK (negated in modes 1 and 2), int32 NJJ, int32 NII, float wind direction, float wind
 * speed, int32 stability class, float DXK, int32 format flag (-1, -2, -3; -1 for the .tke file).
 * Values are int16 of 100 x the field value, clamped to the int16 range.
 *   GRAL_GFF_COLUMNS  flag -1 (GFFWrite.cs:167-254): i = 1..NII+1, j = 1..NJJ+1, k = 1..NKK+1,
 *                     U[k-1], V[k-1], W[k] interleaved per level; truncating conversion.
 *   GRAL_GFF_LEVELS   flag -2 (:256-386): k outer, then rows i, each row U, V, W over j.
 *   GRAL_GFF_TERRAIN  flag -3 (:388-520): KKART of i = 1..NII, j = 1..NJJ, then per column the
 *                     levels k = max(KKART,1)..NKK+1 of U, then V, then W; round-half-even.
 *   GRAL_GFF_TKE      the .tke file of model 2 (:83-133): TURB of i = 1..NII, j = 1..NJJ,
 *                     k = 1..NKK, round-half-even; a non-finite value fails (GRAL_ENONFINITE),
 *                     where the reference's conversion throws and the file is deleted. */
#define GRAL_GFF_COLUMNS 0
#define GRAL_GFF_LEVELS 1
#define GRAL_GFF_TERRAIN 2
#define GRAL_GFF_TKE 3
#define GRAL_GFF_HEADER_BYTES 32

/* Size in bytes of the payload `mode` gives for the loaded grid (mode 2 depends on its KKART). */
int gral_prog_gff_size(gral_ctx *ctx, int32_t mode, uint64_t *bytes);

/* Packs the payload of situation `situation` of the last gral_prog_store on the device from the
 * fields that stay resident there until the next load (the values gral_prog_store returned,
 * after the diagnostic step when post_diagnostic is set), into host memory `out` of `capacity`
 * bytes (at least gral_prog_gff_size). */
int gral_prog_gff_pack(gral_ctx *ctx, int32_t situation, int32_t mode, float wind_dir, float wind_speed,
                       int32_t stability_class, uint8_t *out, uint64_t capacity);

/* Instrumentation: runs the device pack of gral_prog_gff_pack `repeats` times on the stored
 * situation (no copy to the host), with L2 flushed by a 256 MiB device write before each launch,
 * and returns the mean device time of one pack launch in *kernel_ms. */
int gral_prog_gff_pack_timed(gral_ctx *ctx, int32_t situation, int32_t mode, int32_t repeats, double *kernel_ms);

/* Reads a flow-field payload of any of the three formats (GFFRead.cs:181-320) on the device into
 * flat [NII+2][NJJ+2][NKK+2] host arrays uk, vk, wk (the layout of gral_fields): the entries the
 * file holds are set from it (value int16 * 0.01f), those of the terrain format below KKART to 0,
 * all other entries to 0.  The header must match nii, njj, |nkk| and dxk, and in the terrain
 * format the file's KKART must equal `kkart` ([NII+2][NJJ+2], needed only for that format), else
 * GRAL_EINVAL, as the reference rejects such a file.  A format flag other than -1, -2, -3 makes
 * the reference read nothing further and succeed: then the arrays are left untouched and
 * *format is set to that flag.  wind_dir, wind_speed, stability_class and format may be NULL.
 * The context needs no load; the grid must fit its capacity. */
int gral_prog_gff_unpack(gral_ctx *ctx, const uint8_t *payload, uint64_t bytes, int32_t nii, int32_t njj,
                         int32_t nkk, float dxk, const int16_t *kkart, float *uk, float *vk, float *wk,
                         float *wind_dir, float *wind_speed, int32_t *stability_class, int32_t *format);

/* ---- Flow-field set-up of the callers (MicroscaleFlat.cs, ReadGeometryAndDomains.cs,
 * ReadVegetation.cs), computed on the device.  The context needs no load; grids must fit its
 * capacity.  Arrays are flat in the layout of gral_static / gral_fields. ---- */

/* Prognostic sub-domains (ReadGeometryAndDomains.cs:321-347): ADVDOM = 1 in the rectangle
 * i +- (int)(factor*CUTK/DXK), j +- (int)(factor*CUTK/DYK) around every cell with CUTK > 0,
 * clipped to 1..NII x 1..NJJ, 0 elsewhere.  factor = Program.PrognosticSubDomainFactor. */
int gral_prog_subdomains(gral_ctx *ctx, int32_t nii, int32_t njj, float dxk, float dyk, int32_t factor,
                         const float *cutk, uint8_t *advdom);

/* Met input of one weather situation as MicroscaleFlat.Calculate reads it. */
typedef struct {
    int32_t n_heights;               /* Program.MetProfileNumb (>= 1) */
    const float *measurement_height; /* Program.MeasurementHeight, entries 1..n_heights */
    const float *obs_u, *obs_v;      /* Program.ObsWindU/V, entries 1..n_heights */
    float ob_length;                 /* Program.Ob[1][1] */
    const float *ol_column;          /* Program.OLGral [NII+2][NJJ+2] when AdaptiveRoughnessMax > 0,
                                        else NULL (every column uses ob_length) */
} gral_met;

typedef struct {
    int32_t nii, njj, nkk, vert_cells_ff;
    float dxk, dyk;
    int32_t near_wall; /* damping near obstacle walls (MicroscaleFlat.cs:201-357): 0 none; 1 on columns
                          with ADVDOM == 0 (prognostic approach, SubDomainDistance < 10000); 2 on
                          every column (diagnostic approach) */
    int32_t igeb;      /* Program.IGEB (max((int)(20/DXK), 1)): search range of the damping in cells */
} gral_flat_grid;

/* Flat-terrain set-up of one weather situation before the flow-field solve (MicroscaleFlat.cs:
 * 29-357): KKART, AHK (= BUI_HEIGHT) and KADVMAX from CUTK, the initial U and V from the met
 * profile (power law below the first measurement height and, with one height, above it; linear
 * interpolation between heights), zero inside and on the faces of obstacles, W = 0, the copies
 * to the east and north edge columns, then the optional near-wall damping.  Outputs: kkart, ahk
 * [NII+2][NJJ+2]; *kadvmax; f->uk, vk, wk [NII+2][NJJ+2][NKK+2] (levels 1..NKK of columns 1..NII+1
 * x 1..NJJ+1 as the reference sets them, every other entry 0, which the solve leaves at 0).
 * The order is the reference's sequential one (its parallel loop races on the edge copy).
 * advdom is read only for near_wall == 1.  MathF.Pow/Log values are tabulated on the host with
 * the C library, as .NET evaluates them. */
int gral_prog_flat_init(gral_ctx *ctx, const gral_flat_grid *g, const float *cutk, const float *dzk,
                        const float *hokart, const uint8_t *advdom, const gral_met *met, int16_t *kkart,
                        float *ahk, int32_t *kadvmax, gral_fields *f);

/* One coordinate line of vegetation.dat with the parameters of its area (ReadVegetation.cs:66-82). */
typedef struct {
    double crown_height;  /* m */
    double trunk_height;  /* m: trunk percentage x crown height x 0.01 */
    double trunk_lad, crown_lad;  /* leaf-area densities */
    double cov;           /* cover: percentage x 0.01 */
    int32_t i, j;         /* IXCUT, IYCUT; lines outside 1..NII x 1..NJJ are skipped */
    int32_t drag;         /* 1: rasterised into VEG (isCloser); 0: sets COV only */
    int32_t reserved;
} gral_veg_point;

/* Vegetation rasterisation (ReadVegetation.cs:83-118), the points applied in file order: per
 * point with drag, VEG[i][j][k] for k = KKART-1..NKK-1 by the crown/trunk rule, then COV[i][j].
 * Outputs veg [NII+2][NJJ+2][NKK+2] (0 where no point sets it), veg_mask (1 where the reference
 * allocates VEG[i][j]), cov (in/out: cells without a point keep their value). */
int gral_prog_vegetation(gral_ctx *ctx, int32_t nii, int32_t njj, int32_t nkk, const int16_t *kkart,
                         const float *dzk, const float *hokart, int32_t n_points, const gral_veg_point *points,
                         float *veg, uint8_t *veg_mask, float *cov);

/* ---- Wind at particle positions (Zeitschleife.IntWindCalculate, Intwind.cs:31-152) ---- */

/* Grid constants of the interpolation. */
typedef struct {
    int32_t terrain;    /* 1: Program.Topo == TerrainAvailable (binary search of the level above
                           AHMIN); 0: flat terrain */
    int32_t buildings;  /* flat terrain: Program.BuildingsExist (1: interpolate the flow field;
                           0: the met profile, no flow field) */
    int32_t ikooa, jkooa; /* Program.IKOOAGRAL, JKOOAGRAL: south-west corner of the grid (m) */
    float dxk, dyk;
    float ahmin;        /* Program.AHMIN (terrain) */
    const gral_met *met; /* flat terrain without buildings: the met profile (ol_column unused) */
} gral_wind_grid;

/* One particle: its cell (FFCellX/Y, 1..NII x 1..NJJ), surface height AHint and position. */
typedef struct {
    double x, y;        /* xcoord_nteil, ycoord_nteil (m) */
    float z;            /* zcoord_nteil (m) */
    float ahint;        /* AHint */
    int32_t i, j;       /* IndexI, IndexJ */
} gral_particle;

/* U, V, W and the level index IndexK at n particles, interpolated from the fields of situation
 * `situation` of the last gral_prog_store (resident on the device until the next load), exactly
 * as IntWindCalculate does; dzk and hokart are DZK and HOKART [NKK+2].  A particle whose cell lies
 * outside 1..NII x 1..NJJ gets NaN and the call returns GRAL_EINVAL (the reference would index
 * outside its arrays).  In the profile branch (flat, no buildings) the power law is evaluated
 * with a double-precision pow rounded to float, which can differ from the C library's powf by one
 * unit in the last place (U and V then by up to two); every other result is bit-identical to the
 * reference's float/double evaluation. */
int gral_prog_wind_at(gral_ctx *ctx, int32_t situation, const gral_wind_grid *g, const float *dzk,
                      const float *hokart, int32_t n, const gral_particle *particles, float *ux, float *uy,
                      float *uz, int32_t *index_k);

/* gral_prog_load with the initial U, V, W of every situation built on the device from its met
 * profile met[b] by the flat-terrain set-up of gral_prog_flat_init (grid g, the same for all
 * situations and equal to the parameters' grid), so that a batch needs no host-built field and
 * copies none to the device.  f[b].uk, vk, wk are not read: gral_prog_store writes the results
 * there.  TURB/TDISS of models 0 and 2 are read from f as by gral_prog_load.  p[b].kadvmax and
 * s->kkart must be those of the set-up (gral_prog_flat_init returns them). */
int gral_prog_load_flat(gral_ctx *ctx, int32_t n, const gral_params *p, const gral_static *s, const gral_met *met,
                        const gral_flat_grid *g, gral_fields *f);

/* Instrumentation: device time in ms of the kernels of the last gral_prog_subdomains,
 * gral_prog_flat_init, gral_prog_vegetation or gral_prog_wind_at call on this context (CUDA
 * events around its launches, host copies excluded). */
int gral_prog_prep_last_ms(gral_ctx *ctx, double *kernel_ms);

/* ---- Discrete adjoint of the unrolled SIMPLE iterations (vector-Jacobian product) ----
 *
 * Differentiates the map that PrognosticFlowfield.Calculate (PrognosticFlowfield.cs:584-1137)
 * applies to one situation's initial U, V, W and its vegetation density VEG over a fixed number
 * of iterations, in the configuration turbulence_model = 1, simd_width = 8, quantise = 0 (the Frund
 * rounding has derivative zero almost everywhere).  The set-up's scalars (topwind, DTIME, AP0,
 * UG, VG, the wall-law help terms) are constants of the map; kinks of max/min/abs follow the
 * branch the forward takes.  Every wait of the reverse sweeps is bounded (GRAL_ETIMEDOUT). */

/* Runs `iterations` SIMPLE iterations of one situation (p, s, f as for gral_prog_solve; p's
 * iteration limits are replaced by `iterations`, post_diagnostic is ignored), keeping the state
 * every `checkpoint_every` iterations on the device, and writes the final fields to f.  The
 * checkpoints stay for gral_prog_vjp until the next load of the context; gral_prog_vjp recomputes
 * each segment from its checkpoint.  checkpoint_every = 0 keeps instead every iteration's states
 * (ten fields of (NII+2)*(NJJ+2)*KS floats per iteration, KS = KADVMAX+2 rounded up to a multiple
 * of 8: 52 MB on a 200x200 grid with KS 32, plus the boundary-copy branches), and gral_prog_vjp
 * recomputes nothing
 * (GRAL_ENOMEM when they do not fit).  GRAL_EINVAL for another model, parity width or rounding, a
 * batched layout, or a negative spacing. */
int gral_prog_vjp_forward(gral_ctx *ctx, const gral_params *p, const gral_static *s, gral_fields *f,
                          int32_t iterations, int32_t checkpoint_every);

typedef struct gral_vjp_stats {
    int32_t iterations, checkpoint_every;
    double ms_forward;     /* device time of the forward run in gral_prog_vjp_forward */
    double ms_recompute;   /* device time of the segment recomputations inside gral_prog_vjp (each but
                              the last segment's runs beside the reverse sweeps of the segment after it) */
    double ms_reverse;     /* device time of the reverse sweeps */
    double ms_total;       /* device time of gral_prog_vjp (less than recompute + reverse: they overlap) */
} gral_vjp_stats;

/* The vector-Jacobian product of the last gral_prog_vjp_forward: given the cotangents dJ/dUK,
 * dJ/dVK, dJ/dWK of its final fields ([NII+2][NJJ+2][NKK+2] host arrays, NULL = zero), writes
 * dJ/dVEG (same layout; zero where VEG[i][j] is null) and dJ/d(initial UK, VK, WK) (same layout).
 * Any output may be NULL.  The checkpoint segments are recomputed from the kept states (each
 * segment once, the next one on a second stream of the context while the current one is reversed,
 * so two segments' states are held), and the fields resident on the device afterwards are those of
 * an intermediate iteration.  stats may be NULL. */
int gral_prog_vjp(gral_ctx *ctx, const float *dj_duk, const float *dj_dvk, const float *dj_dwk, float *dj_dveg,
                  float *dj_duk0, float *dj_dvk0, float *dj_dwk0, gral_vjp_stats *stats);

/* Text of the last error on this context (never NULL). */
const char *gral_prog_last_error(gral_ctx *ctx);

/* Release the context and its device memory. */
void gral_prog_destroy(gral_ctx *ctx);

/* No counterpart in the reference.  Allocation-free unrealistic-wind-speed check of a solved flow
 * field that already lives on the GPU: the same counts gral_prog_store reports (uk/vk/wk
 * _unrealistic: per ADVDOM==1 column, levels 1..min(NKK-1, KKART+vert_cells_ff), |U| or |V| above
 * 55 m/s, |W| above 20 m/s, or any of them above 10*geschw_max) plus the number of cells holding a
 * non-finite U, V or W, in counts[0..3].
 *
 * For callers that cannot call cudaMalloc when they run the check: a host whose device memory is
 * committed to its own pool (a cudaMalloc would fail or make that pool give memory back) or that
 * must not let cudaMalloc/cudaFree synchronise the device while its other streams run.  It needs
 * no context: uk/vk/wk ([NII+2][NJJ+2][NKK+2]), advdom and kkart ([NII+2][NJJ+2]) are device
 * pointers in the host layout above, counts is host memory, stream a cudaStream_t (NULL: the
 * legacy default stream) on the current device.  The call allocates no memory; its scratch is a
 * fixed static device array of GRAL_NOALLOC_MAX_ROWS rows (64 KiB + 256 B per device that loads
 * the library, held until the process exits), so nii above GRAL_NOALLOC_MAX_ROWS returns
 * GRAL_ETOOLARGE.  Host pointers and device memory of a GPU other than the current one return
 * GRAL_EINVAL; an error already pending in the CUDA runtime on entry returns GRAL_ECUDA and is
 * left pending for the caller.  The first call on a device looks up that array's device address
 * (with the device current) and keeps it for the life of the process, so do not call it on a
 * device after cudaDeviceReset of that device.  Never call it while `stream` is capturing, nor
 * while any stream is capturing in the global capture mode: every call copies the counts into
 * pageable host memory and synchronises `stream`, which fails under capture (and in the global
 * mode can invalidate another thread's capture).  All calls on a device share the array, so calls
 * that overlap on the GPU (two host threads, or two streams) race and may return wrong counts:
 * serialise them.  The call synchronises `stream` and returns after the counts are on the host. */
#define GRAL_NOALLOC_MAX_ROWS 4096
int gral_prog_check_speeds_noalloc(int32_t nii, int32_t njj, int32_t nkk, int32_t vert_cells_ff,
                                   double geschw_max, const float *uk, const float *vk,
                                   const float *wk, const uint8_t *advdom, const int16_t *kkart,
                                   int32_t counts[4], void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GRAL_PROG_H */
