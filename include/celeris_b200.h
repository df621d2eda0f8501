/*
 * celeris_b200.h — C ABI of the B200-native Celeris Boussinesq timestep path.
 *
 * Drop-in boundary for the reference's `class ShallowWaterEngine` (engine.hpp:58-312):
 * one `cel_engine` handle equals one engine (one simulated domain) with its own CUDA stream.
 * Parameters come in as a `cel_params` value (the fields readInputCML fills from a `.cml`
 * file, main.cpp:500-913) instead of the reference's `initSetting` / `GetSetting` globals.
 *
 * Conventions
 *   - Every function returns `int` status: 0 = CEL_OK, non-zero = error; the message is
 *     available from `cel_last_error()` (thread-local).  No C++ exception crosses the ABI.
 *   - Host buffers are owned by the caller; device memory is owned by the library.
 *   - Grid arrays use the reference texture layout: (nx+4) x (ny+4) texels with two ghost
 *     cells per side, row-major `y*(nx+4)+x` (engine.cpp:413-489).  State texels are
 *     {w = eta + still water level, hu, hv, unused} (compute.hlsl:160-164); bottom texels are
 *     {BY, BX, BA} (terrain_heightfield.hpp:50-52).
 *   - A handle is not thread-safe; distinct handles may be used concurrently.
 *   - The library never falls back to a CPU path: without a CUDA device every call that
 *     needs one returns CEL_ERR_CUDA.
 */
#ifndef CELERIS_B200_H
#define CELERIS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CEL_OK 0
#define CEL_ERR_ARG 1        /* invalid argument / size */
#define CEL_ERR_IO 2         /* file missing or malformed */
#define CEL_ERR_CUDA 3       /* CUDA runtime error or no device */
#define CEL_ERR_STATE 4      /* call not valid in the handle's current state */
#define CEL_ERR_NUMERIC 5    /* device health flag: NaN or Inf in the state (a cell below its bed is dry, not an error) */

#define CEL_MAX_WAVES 1000   /* MAX_NUM_OF_IRREGULAR_WAVES (engine.hpp:214) */
#define CEL_MAX_SOLITONS 100 /* InitSetting::MAX_NUM_SOLITARY (settings.hpp:356) */
#define CEL_MAX_CR_LEVELS 15 /* ST_MAX_CR_MATRIX_NUM_X/Y (engine.hpp:173-176) */

/* Boundary types (settings.hpp:99-105; the .cml `type` string) */
#define CEL_BC_SOLID 0
#define CEL_BC_SPONGE 1
#define CEL_BC_SINEWAVE 2
#define CEL_BC_IRREGULAR 3
#define CEL_BC_UTS 4

/* Solver forms */
#define CEL_FORM_PLAIN 0  /* FP32, one kernel per reference pass and per CR level */
#define CEL_FORM_FUSED 1  /* FP32, fused stencil + Thomas factors solved as scans */
#define CEL_FORM_MIXED 2  /* fused, compensated (two-sum) state, FP64 clock and reductions */

/* Time schemes (settings.hpp:298: enum TimeIntegrationScheme) */
#define CEL_SCHEME_EULER 0
#define CEL_SCHEME_PREDICTOR 1
#define CEL_SCHEME_CORRECTOR 2
#define CEL_SCHEME_PREDICTOR_ADAPTIVE 3

typedef struct cel_boundary {
    int type;                 /* CEL_BC_* */
    int width;                /* widthNum: cells in the boundary strip */
    double sea_level;         /* seaLevel */
    double amplitude;         /* SineWave amplitude (m) */
    double period;            /* SineWave period (s) */
    double theta;             /* SineWave direction (radians; the .cml gives degrees) */
    int n_waves;              /* IrregularWaves component count (<= CEL_MAX_WAVES) */
    double waves[CEL_MAX_WAVES][4]; /* amplitude, period, theta (rad), phase */
    int n_uts;                /* UniformTimeSeries rows */
    double* uts;              /* n_uts x {t, eta, hu, hv}; owned by the cel_params */
} cel_boundary;

typedef struct cel_soliton {
    double H, theta, xc, yc, length; /* theta in radians; length 1e30 = infinite crest */
} cel_soliton;

/* Run-time logging of the `.cml` <logData> element (main.cpp:825-887; InitSetting fields and
 * defaults settings.hpp:322, 359-372, 389, 423-433).  Indices are texel indices of the
 * (nx+4) x (ny+4) layout, ghost cells included, as the reference's staging-texture reads use them. */
#define CEL_MAX_LOG_RANGES 100  /* InitSetting::MAX_NUM_RANGE (settings.hpp:362) */
#define CEL_MAX_GAUGES 1000     /* InitSetting::MAX_NUM_GAUGE (settings.hpp:368) */

typedef struct cel_log_range {
    char name[256];           /* range `filename`: rows go to <path>/<name>.txt */
    int x0, y0;               /* bottomLeft x, y */
    int x1, y1;               /* topRight x, y (inclusive) */
} cel_log_range;

typedef struct cel_log {
    int do_log;               /* logData doLog (default 0) */
    int log_step;             /* logData logStep: log after every log_step-th physical step (default 100) */
    char path[1024];          /* logPath, resolved against the .cml folder (default "NA") */
    char time_axis_name[256]; /* timeAxis filename (default "time_axis") */
    char gauges_name[256];    /* gauges filename (default "gauges") */
    int n_ranges;
    cel_log_range ranges[CEL_MAX_LOG_RANGES];
    int n_gauges;
    int gauges[CEL_MAX_GAUGES][2];  /* {x, y} per gauge */
} cel_log;

typedef struct cel_params {
    int nx, ny;                       /* gridSize */
    double width, length;             /* fieldDimensions (x, y extent in m) */
    double still_water_elevation;     /* fieldDimensions stillWaterElevation */
    int boussinesq;                   /* model type BSNQ (1) / NLSW (0) */
    double epsilon, theta;            /* parameters epsilon, Theta */
    int correction_steps;             /* parameters correctionStepsNum */
    double timestep;                  /* parameters timestep */
    int adaptive;                     /* parameters adaptive */
    double ema_alpha;                 /* parameters exponentialMovingAverageAlpha */
    double min_timestep_ratio;        /* InitSetting::min_timestep_ratio */
    int manning;                      /* friction type Manning (1) / Quadratic (0) */
    double friction;                  /* friction coef */
    double gravity;                   /* 9.81 (gui_manager.cpp:106) */
    double dissipation_threshold;     /* graphics dissipationIntensity threshold */
    double whitewater_decay;          /* graphics dissipationIntensity decay */
    cel_boundary west, east, south, north;
    int n_solitons;
    cel_soliton solitons[CEL_MAX_SOLITONS];
    char bathymetry_path[1024];       /* bathymetryFilePath, resolved against the .cml folder */
    char hotstart_path[1024];         /* hotStartFilePath, resolved; "" if none */
    char project_name[256];
    cel_log log;                      /* logData */
} cel_params;

/* resetTimestep() outputs (engine.cpp:1685-1746), reduced on the device in FP64. */
typedef struct cel_stats {
    double mass, x_momentum, y_momentum;
    double kinetic_energy, potential_energy, total_energy;
    double max_speed, max_depth, max_froude;
    double cfl_rate;      /* max((|u|+c)/dx, (|v|+c)/dy) */
    double cfl_number;    /* cfl_rate * dt */
    double timestep;      /* dt for the next pass */
    double total_time;    /* simulated time */
    double mass_full;     /* sum of h over every interior cell (FP64), m */
    int time_scheme;      /* scheme of the next pass (CEL_SCHEME_*) */
    int health;           /* 0 = ok, else CEL_ERR_NUMERIC */
} cel_stats;

typedef struct cel_engine cel_engine;
typedef struct cel_batch cel_batch;

/* ---- errors ---------------------------------------------------------------------------- */
const char* cel_last_error(void);
const char* cel_version(void);

/* ---- parameters ------------------------------------------------------------------------- */
/* InitSetting defaults (settings.hpp:370-438); replaces `InitSetting()` */
int cel_params_default(cel_params* p);
/* readInputCML (main.cpp:500-913): lenient XML (unquoted attributes, comments).  Irregular
 * wave and uniform-time-series files named in the .cml are read too (engine.cpp:3512-3560,
 * 3863-3909).  Free with cel_params_release. */
int cel_params_from_cml(const char* path, cel_params* out);
/* Reads an IrregularWaves component file into a boundary (engine.cpp:3520-3551) */
int cel_read_irregular_waves(const char* path, cel_boundary* b);
/* Spectrum wave-maker settings (IrregularWaveSpectrumSetting, settings.hpp:121-129; set from
 * the GUI's "significant waveheight", "peak period", "mean direction", "depth at source") */
typedef struct cel_spectrum {
    double significant_waveheight;  /* Hs (m), capped at half the source depth */
    double peak_period;             /* Tp (s) */
    double mean_theta;              /* mean direction (degrees) */
    double depth_at_source;         /* h (m) */
} cel_spectrum;
/* generateSpectrumWaves (engine.cpp:3559-3776): JONSWAP-shaped spectrum (gamma 3.3) on
 * f_peak +- 5 x 0.005 Hz, cos^2s spreading over mean +- 20 degrees in 5-degree steps, truncated
 * at 5 % of the peak; one component {amplitude, period, theta (rad), phase} per (f, theta) cell
 * into b->waves / b->n_waves.  Phases come from `seed` (the reference seeds rand() with the
 * clock), quantised as (r % 10000) / 10000 x 2 pi.  path != NULL also writes the reference's
 * component file, which cel_read_irregular_waves reads back. */
int cel_spectrum_waves(const cel_spectrum* s, double gravity, unsigned long long seed, cel_boundary* b,
                       const char* path);
/* Reads a UniformTimeSeries file into a boundary (engine.cpp:3863-3874) */
int cel_read_uts(const char* path, cel_boundary* b);
void cel_params_release(cel_params* p);
/* sizeof(cel_params), for bindings that mirror the struct */
size_t cel_params_size(void);

/* Reads a .cbf bathymetry grid (terrain_heightfield.cpp:136-209).  If z is NULL, only the
 * header size is returned. */
int cel_read_cbf(const char* path, float* z, size_t capacity, int* bnx, int* bny);

/* ---- engine lifecycle (ShallowWaterEngine ctor + remesh, engine.cpp:709-737) ------------- */
/* bathy: bnx*bny row-major grid spanning x in [-W/2, W/2], y in [0, L] (the .cbf content);
 * NULL = read params->bathymetry_path.  Builds the staggered bottom, the tridiagonal
 * coefficients and the initial condition (hot start + solitary waves) and uploads them. */
int cel_create(const cel_params* p, const float* bathy, int bnx, int bny, int form, cel_engine** out);
int cel_destroy(cel_engine* h);
int cel_remesh(cel_engine* h);   /* remesh(R_MESH): back to the initial condition, Euler bootstrap */
int cel_set_stream(cel_engine* h, void* cuda_stream);   /* NULL = the library's own stream */
int cel_get_dims(const cel_engine* h, int* nx, int* ny);

/* ---- state import/export in the reference layout ---------------------------------------- */
int cel_set_state(cel_engine* h, const float* rgba);      /* (nx+4)(ny+4) x {w,hu,hv,_} */
int cel_get_state(cel_engine* h, float* rgba);
int cel_get_bottom(cel_engine* h, float* by_bx_ba);      /* (nx+4)(ny+4) x {BY,BX,BA} */
int cel_get_aux(cel_engine* h, float* rgba);             /* txAuxiliary1: {maxdepth,0,0,breaking} */

/* ---- the step (engine.hpp:64-93) --------------------------------------------------------- */
/* resetTimestep(realworld_dt, elapsed): stats of the current state, then dt for the next pass */
int cel_reset_timestep(cel_engine* h, float realworld_dt, float elapsed, cel_stats* out);
/* timestep(): one pass (Euler, AB3 predictor or AM4 corrector) */
int cel_timestep(cel_engine* h);
/* n passes, each preceded by the device-side resetTimestep (no host readback) */
int cel_timesteps(cel_engine* h, int n);
/* n physical steps (a predictor/Euler pass plus its correctors), device-side stats */
int cel_physical_steps(cel_engine* h, int n);
/* latest device-side stats (copies to host; synchronizes the stream) */
int cel_get_stats(cel_engine* h, cel_stats* out);
/* addSolitaryWave (engine.cpp:2154-2219, AddSolitaryWave pass compute.hlsl:949-976): adds a sech^2
 * wave of height H, direction theta_deg and centre (xc, yc) (texel-index coordinates x dx, y dy)
 * to the current state, each texel with its own water depth. */
int cel_add_solitary_wave(cel_engine* h, double H, double theta_deg, double xc, double yc);
/* getWaterHeight (engine.cpp:4994-5012): the water surface at world point (x, y), x in
 * [-W/2, W/2], y in [0, L], as the terrain height there (GetTerrainHeight, a float bilinear of BA)
 * plus the mean depth of the GetStats 4x4 block holding the point.  The plain form takes the block
 * from its latest GetStats (the state of the latest resetTimestep), as the reference reads its
 * staging texture; the fused forms sum the block of the current state.  Points on the far edges
 * use the last block (the reference reads past its block array there). */
int cel_get_water_height(cel_engine* h, float x, float y, float* out);
int cel_synchronize(cel_engine* h);
/* newTerrainSettings (engine.hpp:63, engine.cpp:820-823 -> fillTerrainTexture 3313-3379): a new
 * bathymetry grid (bnx x bny, the .cbf layout) replaces the bottom.  Every texel keeps its water
 * depth (w - BA_old + BA_new), both aux textures are cleared and the next pass re-bootstraps.  As
 * in the reference, the tridiagonal coefficients keep the old bottom until cel_remesh, which
 * rebuilds everything (coefficients, initial condition) from the new grid. */
int cel_set_bathymetry(cel_engine* h, const float* bathy, int bnx, int bny);

/* ---- batched ensembles: many domains advanced by one launch per phase ------------------- */
/* params[i] and bathy[i] (bnx[i] x bny[i]) describe member i; form is CEL_FORM_FUSED or
 * CEL_FORM_MIXED.  Members share correctionStepsNum and the adaptive setting.  Adaptive batches
 * choose each member's dt on the device before every pass, as resetTimestep does
 * (engine.cpp:1698-1726: target CFL from the first positive CFL rate, moving-average growth,
 * uniform dt for Euler and corrector passes) and run the variable-step AB3 predictor
 * (compute.hlsl:766-780); a step needs no host readback and replays from a CUDA graph. */
int cel_batch_create(int n, const cel_params* const* params, const float* const* bathy,
                     const int* bnx, const int* bny, int form, cel_batch** out);
/* cel_batch_create with the member set split into `lanes` lanes (0 = the default: 2 for two or
 * more members).  Each lane is advanced by its own launches and CUDA graphs on its own stream,
 * ordered against the batch stream at every call; lanes run side by side, so one lane's small
 * boundary launches and kernel tails overlap another lane's stencil.  Members are assigned by
 * interior cell count (largest first, to the lane with the fewest cells); results do not depend
 * on the split.  No counterpart in the reference. */
int cel_batch_create_lanes(int n, const cel_params* const* params, const float* const* bathy,
                           const int* bnx, const int* bny, int form, int lanes, cel_batch** out);
int cel_batch_lanes(const cel_batch* b);                 /* lanes of a batch (0 for NULL) */
int cel_batch_destroy(cel_batch* b);
int cel_batch_set_stream(cel_batch* b, void* cuda_stream);
int cel_batch_step(cel_batch* b, int nsteps);            /* physical steps, all members */
/* n entries: the GetStats totals (FP64) of each member's state at the start of the most recent
 * step, gathered by that step's first pass as the reference's resetTimestep gathers them before a
 * step (engine.cpp:1536-1756); total_time is that start time.  Before any step (or after
 * cel_batch_set_state) they are computed from the current state. */
int cel_batch_stats(cel_batch* b, cel_stats* out);
/* n entries: the same totals computed now, from the current state (one extra pass over it). */
int cel_batch_stats_current(cel_batch* b, cel_stats* out);
int cel_batch_get_state(cel_batch* b, int i, float* rgba);
/* Member i's state as two RGBA32F textures whose sum is the compensated state of the mixed form:
 * hi (the stored state, what the stencils read) and lo (its low words; 0 in the FP32 forms).
 * cel_batch_get_state returns hi + lo rounded to float.  Either pointer may be NULL.  Library only. */
int cel_batch_get_state_parts(cel_batch* b, int i, float* hi_rgba, float* lo_rgba);
int cel_batch_set_state(cel_batch* b, int i, const float* rgba);
int cel_batch_get_aux(cel_batch* b, int i, float* rgba);
/* cel_add_solitary_wave for member i */
int cel_batch_add_solitary_wave(cel_batch* b, int i, double H, double theta_deg, double xc, double yc);
/* cel_set_bathymetry for member i (the member's Thomas factors keep the old bottom). */
int cel_batch_set_bathymetry(cel_batch* b, int i, const float* bathy, int bnx, int bny);
int cel_batch_use_graph(cel_batch* b, int enable);        /* capture one physical step in a CUDA graph */
long long cel_batch_cells(const cel_batch* b);            /* sum of interior nx*ny */
/* Per-member uniform time step (n floats), uploaded asynchronously on the batch stream; the
 * reference uploads dt with its constant buffers before every pass (engine.cpp:1728-1750).
 * CEL_ERR_STATE for adaptive batches, which choose their steps on the device. */
int cel_batch_set_timestep(cel_batch* b, const float* dt);
/* Kernel launches one physical step issues (all members together). */
int cel_batch_launches_per_step(const cel_batch* b);

/* ---- tuning and measurement ------------------------------------------------------------- */
/* Fused forms.  tile_x: column-solver band width (8, 16 or 32 columns per CTA, chunked scans; or 1:
 * one thread per column, serial sweeps, forward values kept in the right-hand-side plane); tile_y: stencil
 * strip height (rows a CTA marches, 8..1024); 0 keeps the current value.  pcr_switch: chunks per
 * column of the column solver, i.e. where it switches from the parallel stage to serial sweeps.  The
 * solves factor each system once (M = LU, engine.cpp:2612-2887 coefficients); the L and U sweeps of
 * a column are split into that many chunks, each swept serially by one thread (Thomas), and the
 * chunks' transfer maps are joined by recursive doubling with warp shuffles (parallel reduction of
 * the bidiagonal sweeps).  Chunks x band width must be 256 or 512 threads, or, with tile_x = 32, 32,
 * 64 or 128 chunks: the cluster solver, where a cluster of chunks/8 CTAs holds a 32-column band with
 * every chunk (at most 16 rows, so the tallest member must have at most 16 x chunks rows) in
 * registers and joins the chunks' maps through distributed shared memory; or, with tile_x = 16,
 * 1 chunk: the tile-transposed solver, where a warp sweeps each column of 128-row tiles staged
 * through shared memory by the CTA; 0 keeps the current value.  Plain engines ignore the call. */
int cel_set_tuning(cel_engine* h, int tile_x, int tile_y, int pcr_switch);
int cel_batch_set_tuning(cel_batch* b, int tile_x, int tile_y, int pcr_switch);
int cel_batch_get_tuning(const cel_batch* b, int* tile_x, int* tile_y, int* rows_per_step);
/* The column solver's chunks per column (the pcr_switch above; 1 with tile_x = 1: one thread per column). */
int cel_batch_col_chunks(const cel_batch* b);
/* Stencil variant: 1 = one row per thread step; 2 = two rows per step as pairs, with the paired
 * single-precision instructions of sm_100 (f32x2). */
int cel_batch_set_stencil_rows(cel_batch* b, int rows_per_step);
/* Threads per stencil CTA, i.e. strip width + 2 halo columns: 128 or 96 (96 with two rows per step
 * only).  Narrower strips waste fewer lanes on members whose width is not a multiple of 126. */
int cel_batch_set_stencil_width(cel_batch* b, int threads);
int cel_batch_stencil_width(const cel_batch* b);
/* Times `steps` physical steps for each candidate (band width x strip height x stencil rows per
 * step x stencil width) and keeps the fastest; writes the choice and its ms per step.  The
 * members advance by every timed step. */
int cel_batch_autotune(cel_batch* b, int steps, int* tile_x, int* tile_y, double* ms_per_step);
/* Per-kernel CUDA-event timing on the launching stream (off by default). */
int cel_batch_kernel_timing(cel_batch* b, int enable);
int cel_engine_kernel_timing(cel_engine* h, int enable);
/* Copies up to cap (name, total ms, launches) records; returns the count in *n. */
int cel_kernel_times(void* handle, int is_batch, char (*names)[64], double* total_ms, long long* launches,
                     int cap, int* n);
/* Device self-test of the fused forms' flux reciprocal (no counterpart in the reference): writes
 * to out[i] what the Kurganov-Petrova flux uses as 1 / x[i] (the hardware approximation refined by
 * one Newton-Raphson step), computed on the current device; x and out are host arrays of n floats.
 * It allocates device memory for the call. */
int cel_selftest_reciprocal(const float* x, float* out, int n);
/* Algorithmic HBM bytes per cell for one pass of the dominant kernel and for a whole
 * physical step (the roofline byte model recorded in code). */
int cel_byte_model(int form, int correction_steps, double* stencil_bytes_per_cell_pass,
                   double* step_bytes_per_cell);

/* ---- logging and file output (host side; no device needed) ------------------------------ */
/* Engines and batch members whose params have log.do_log set log by themselves, as the reference's
 * timestep() does (engine.cpp:1488-1493): after physical step s with s % log_step == 0 the state
 * after that step is written as below, with the simulated time at the start of that step (the
 * reference writes total_time before adding the step's dt, engine.cpp:1491-1518).  The elapsed
 * time is the `elapsed` argument of the engine's latest cel_reset_timestep call (0 before one; the
 * reference writes its "elapsed time" setting, which resetTimestep sets, engine.cpp:1746); batch
 * members write the wall-clock seconds since the batch was created.  A failed write makes the
 * stepping call return CEL_ERR_IO after the step has completed.  Creation fails with CEL_ERR_ARG
 * if a gauge or a non-empty range lies outside the texture, or log_step < 1 with do_log set. */

/* st_DumpToFile (engine.cpp:628-675) for a host state rgba ((nx+4)(ny+4) x {w,hu,hv,a}):
 * appends total_time to <path>/<time_axis_name>.txt and elapsed to <path>/<time_axis_name>-elapsed.txt,
 * then "i\tj\tw\thu\thv\ta\n" for each texel of each range (j outer, i inner) to <path>/<name>.txt
 * and for each gauge to <path>/<gauges_name>.txt; numbers in the default stream format (6
 * significant digits). */
int cel_log_dump(const cel_params* p, const float* rgba, float total_time, float elapsed);
/* dumpInundationToFile (engine.cpp:781-817): the maximum-inundation-depth map from an aux array
 * (cel_get_aux layout, component 0) with the reference's "[nx]/[ny]" header; rows j = 2..ny+1,
 * columns i = 2..nx+2 (one ghost column included, as the reference writes it).  path NULL =
 * <log path>/<Y-M-D H-M-S>-inundation.txt in local time, as the reference names it. */
int cel_write_inundation(const cel_params* p, const float* aux_rgba, const char* path);
/* dumpBathymetryToFile (engine.cpp:750-779): the interior cell bottom (BA of a cel_get_bottom
 * array) as a .cbf text grid.  path NULL = <log path>/<Y-M-D H-M-S>.cbf. */
int cel_write_bathymetry(const cel_params* p, const float* bottom_b3, const char* path);
/* A hot-start file for hotStartFilePath (read by engine.cpp:2943-2966): "i j w hu hv a" per texel
 * over all (nx+4)(ny+4) texels, j outer, with 9 significant digits so that the state reads back
 * bit for bit (the reference's range dump writes the same columns with 6). */
int cel_write_hotstart(const cel_params* p, const float* rgba, const char* path);

/* ---- allocation-free statistics (no counterpart in the reference) ----------------------- */
/* The resetTimestep statistics (mass, energies, momenta, maxima, CFL rate, the FP64 volume) of a
 * state the caller keeps in device memory: d_state_rgba is (nx+4)(ny+4) x {w,hu,hv,_} and
 * d_bottom_b3 is (nx+4)(ny+4) x {BY,BX,BA}, both device pointers; p supplies nx, ny, width, length,
 * gravity and epsilon.  The work runs on cuda_stream (NULL = the default stream); the call waits
 * for that stream and returns once the totals are in *out.  It never allocates device or pinned
 * memory, for callers that must not allocate when they ask: frame loops where the device-wide
 * synchronisation of cudaMalloc / cudaFree would stall every other stream, and applications whose
 * own allocator has reserved the device's memory.  Its scratch is a fixed static device array
 * (about 2.4 MB on every GPU that loads the library, held until exit) sized for at most 65,536
 * 4x4 blocks, i.e. 1,048,576 interior cells; larger domains get CEL_ERR_ARG.  The first call on
 * each device looks up the array's address.  Every call uses the same array: calls whose work
 * overlaps on the GPU (different streams or threads) race, so run them one after another. */
int cel_stats_noalloc(const float* d_state_rgba, const float* d_bottom_b3, const cel_params* p, void* cuda_stream,
                      cel_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* CELERIS_B200_H */
