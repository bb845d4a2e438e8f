/*
 * speedy_b200.h -- C ABI of the B200 (sm_100a) SPEEDY column physics.
 *
 * The entry points replace the reference's SPEEDY physics call
 *   SpeedyPhysics.compute_tendencies(state, forcing, geometry, date)
 *     (jcm/physics/speedy/speedy_physics.py:88-127)
 * as it is invoked from
 *   get_physical_tendencies (jcm/physics_interface.py:344-383),
 * including the verify_state / verify_tendencies clamps around it
 *   (jcm/physics_interface.py:305-342, fused behind SPD_FUSE_VERIFY).
 *
 * Conventions
 *  - All array arguments are DEVICE pointers owned by the caller; the library never frees them.
 *  - Layout is the reference's: level fields are [kx][ix][il] row-major (column c = i*il + j,
 *    latitude index j = c % il), surface fields [ix][il], latitude tables [il] south->north.
 *  - float32 everywhere (the reference computes in float32).
 *  - Every call is asynchronous on `stream` (a cudaStream_t passed as void*), makes no host
 *    synchronisation and allocates no memory; scratch is caller-provided.
 *  - Return value 0 (SPD_OK) or one of the SPD_ERR_* codes; no exceptions cross the ABI.
 *  - The forward's output fields overlap neither its input fields nor one another
 *    (SPD_ERR_ALIAS): columns write their outputs while other columns still read their
 *    inputs, and a fixup launch (a missed level-set prediction) or the level-set launch
 *    (SPD_NO_SPECULATION) reads the state again.
 */
#ifndef SPEEDY_B200_H
#define SPEEDY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPD_MAX_KX 16
#define SPD_ABI_VERSION 1

enum spd_status {
  SPD_OK = 0,
  SPD_ERR_NULL = 1,      /* a required pointer is NULL */
  SPD_ERR_SHAPE = 2,     /* ix, il, member count or column count out of range */
  SPD_ERR_KX = 3,        /* unsupported level count (supported: 7, 8, 16) */
  SPD_ERR_SCRATCH = 4,   /* scratch buffer NULL, too small or not 256-byte aligned */
  SPD_ERR_CUDA = 5,      /* a CUDA launch or runtime call failed */
  /* 6 is not used: no kernel waits on another or reports a status of its own */
  SPD_ERR_ALIGN = 7,     /* a field pointer is not 16-byte aligned */
  SPD_ERR_NOALLOC_LIMIT = 8, /* il above SPD_NOALLOC_MAX_IL for spd_fwd_noalloc */
  SPD_ERR_ALIAS = 9,         /* an output field overlaps an input field or another output */
  SPD_ERR_STREAM_DEVICE = 10 /* spd_fwd_noalloc: the stream belongs to another device than the
                                current one */
};

/* spd_desc_t.flags */
enum spd_flags {
  SPD_LFLUXLAND = 1u << 0,    /* ForcingData.lfluxland (jcm/forcing.py:17) */
  SPD_LSCASYM = 1u << 1,      /* SurfaceFluxParameters.lscasym (params.py:180) */
  SPD_LSKINEB = 1u << 2,      /* SurfaceFluxParameters.lskineb (params.py:181) */
  SPD_INCREASE_CO2 = 1u << 3, /* ForcingParameters.increase_co2 (params.py:34) */
  SPD_FUSE_VERIFY = 1u << 4,  /* apply verify_state before and verify_tendencies after */
  SPD_OROGRAPHIC = 1u << 5,   /* orographic correction as the last term (orographic_correction.py
                                 :177-247; commented out of the reference's term list at
                                 speedy_physics.py:65,79).  Its tendency divides by
                                 spd_desc_t.dt_seconds, which must then equal
                                 DateData.dt_seconds. */
  SPD_ACCUMULATE_DIAGNOSTICS = 1u << 6,
  /* The forward adds precnv, precls and every non-NULL float diagnostic to what the output
   * buffers hold (out[c] += value) instead of overwriting them; the tendency planes and the
   * integer levels are written as usual.  This is DiagnosticsCollector's running average
   * (jcm/model.py:46-64: data[i] += new / steps) without a pass over PhysicsData per physics
   * step: zero the buffers, make the steps' calls, scale by 1/steps once. */
  SPD_LOW_LEVEL_WINDS = 1u << 7,
  /* Forward only: spd_inputs_t.u_wind / v_wind and spd_outputs_t.u_wind / v_wind are single
   * [ix][il] planes holding the lowest level.  The physics reads the winds at the lowest level
   * only (surface_flux.py:57-58) and its wind tendencies are zero above it (surface_flux.py
   * :294-295), so a caller that keeps those zeros itself moves 2 (kx - 1) fewer planes each
   * way (the reference returns dense [kx][ix][il] planes; the default writes them). */
  SPD_NO_SPECULATION = 1u << 8
  /* Forward only: form the level set of cloud tops before the columns that need it (a light
   * launch over every column, then the fused launch) instead of predicting it from the
   * previous call.  Implied by SPD_ACCUMULATE_DIAGNOSTICS, whose added diagnostics a redone
   * column would add twice.  A caller whose every call is a new instance (a fresh plan per
   * batch) sets it: there is no previous call to predict from. */
};

/* One grid instance: shape, switches and DateData (jcm/date.py:9-14). */
typedef struct {
  int32_t kx, ix, il;
  uint32_t flags;
  float tyear;          /* DateData.tyear */
  int32_t model_year;   /* DateData.model_year */
  int32_t model_step;   /* DateData.model_step: shortwave heating when model_step % 3 == 0 */
  int32_t co2_year_ref; /* ForcingParameters.co2_year_ref */
  float dt_seconds;     /* time step of the fused verify_tendencies limiter */
  float q_tend_scale;   /* factor applied to the humidity tendency last (1 = g/kg/s) */
} spd_desc_t;

/* Vertical sigma tables of Geometry (jcm/geometry.py:62-85, :99-106), by value. */
typedef struct {
  float hsg[SPD_MAX_KX + 1];
  float fsg[SPD_MAX_KX];
  float dhs[SPD_MAX_KX];
  float sigl[SPD_MAX_KX];
  float grdsig[SPD_MAX_KX];
  float grdscp[SPD_MAX_KX];
  float wvi[SPD_MAX_KX][2];
} spd_vgrid_t;

/* The float leaves of Parameters (jcm/physics/speedy/params.py:9-232), by value. */
typedef struct {
  /* ConvectionParameters */
  float psmin, trcnv, rhil, rhbl, entmax, smf;
  /* CondensationParameters */
  float trlsc, rhlsc, drhlsc, rhblsc;
  /* ShortwaveRadiationParameters */
  float albcl, albcls, absdry, absaer, abswv1, abswv2, abscl1, abscl2;
  float ablwin, ablwv1, ablwv2, ablcl1, ablcl2;
  float rhcl1, rhcl2, qacl, wpcl, pmaxcl, clsmax, clsminl, gse_s0, gse_s1;
  /* ModRadConParameters */
  float albsea, albice, albsn, epslw, emisfc;
  /* SurfaceFluxParameters */
  float fwind0, ftemp0, fhum0, cdl, cds, chl, chs, vgust, ctday, dtheta, fstab;
  float clambda, clambsn, hdrag;
  /* VerticalDiffusionParameters */
  float trshc, trvdi, trvds, redshc, rhgrad, segrad;
} spd_params_t;

/* PhysicsState (physics_interface.py:22-29), ForcingData day slice (jcm/forcing.py:8-17)
 * and the per-column / per-latitude Geometry fields (jcm/geometry.py:91-97). */
typedef struct {
  const float *u_wind, *v_wind, *temperature, *specific_humidity, *geopotential; /* [kx][C] */
  const float *normalized_surface_pressure;                                        /* [C] */
  const float *alb0, *sice_am, *snowc_am, *soilw_am, *stl_am, *sea_surface_temperature;
  const float *fmask, *orog, *phis0;                                               /* [C] */
  const float *sia, *coa;                                                          /* [il] */
} spd_inputs_t;

/* PhysicsTendency (physics_interface.py:89-94) plus the PhysicsData leaves the kernel fills.
 * Tendency planes and precnv/precls are required; every other pointer may be NULL. */
typedef struct {
  float *u_wind, *v_wind, *temperature, *specific_humidity; /* [kx][C] */
  float *precnv, *precls;                                    /* [C] */
  float *cbmf, *cloudc, *cloudstr, *rsds, *rsns, *ftop_sw;   /* [C], nullable */
  float *rlds, *rlns, *ftop_lw, *tsfc, *tskin, *shf, *evap;  /* [C], nullable */
  int32_t *iptop, *icltop;                                   /* [C], nullable */
} spd_outputs_t;

/* ----------------------------------------------------------------------------------------- */
/* Plain drop-in: one instance per call.                                                      */
/* ----------------------------------------------------------------------------------------- */

/* Scratch bytes spd_fwd needs for this descriptor (per-instance cloud-top level set, the
 * per-latitude solar tables and a status word). */
size_t spd_fwd_scratch_bytes(const spd_desc_t* desc);

/* SpeedyPhysics.compute_tendencies for one instance (speedy_physics.py:88-127).
 * Two launches on `stream`, each over every column: a light one that forms the instance's
 * cloud-top level set (shortwave_radiation.py:62-68: the cloud tops of every column, from
 * humidity, convection, condensation and clouds) and its per-latitude solar table; then every
 * column whole in one pass (all terms, verify_tendencies when on, every output).  They are the
 * batched kernels below run on a one-member plan, so the results equal the batched path's
 * bitwise.  `scratch` must be 256-byte aligned and at least spd_fwd_scratch_bytes(desc) long;
 * it is initialised by the call. */
int spd_fwd(const spd_desc_t* desc, const spd_vgrid_t* vgrid, const spd_params_t* params,
            const spd_inputs_t* in, const spd_outputs_t* out, void* scratch,
            size_t scratch_bytes, void* stream);

/* Timing hook (no reference counterpart): spd_fwd, recording `event` (a cudaEvent_t, or NULL)
 * on `stream` between its two launches, so that a caller can time them separately with
 * events: after the fused launch (before the fixup) when the call predicts the level set,
 * after the level-set launch (before the fused one) under SPD_NO_SPECULATION.  With an event
 * the launches run in plain stream order; without one (and in spd_fwd) the second launch is a
 * programmatic dependent launch: its blocks start as the first one's retire and wait on the
 * device for the first launch's completion before reading what it wrote. */
int spd_fwd_marked(const spd_desc_t* desc, const spd_vgrid_t* vgrid, const spd_params_t* params,
                   const spd_inputs_t* in, const spd_outputs_t* out, void* scratch,
                   size_t scratch_bytes, void* stream, void* event);

/* Loads every kernel of the library on the current device (no reference counterpart).  CUDA
 * loads modules lazily by default, and loading one while other kernels run waits for them;
 * calling this once per device before latency-sensitive use keeps that wait out of the first
 * launches. */
int spd_preload(void);

/* Self-test of the forward's packed float32 arithmetic (no reference counterpart).  The
 * forward pairs independent float32 operations into sm_100's packed .f32x2 instructions; this
 * evaluates every packed piece on n seeded inputs per piece and compares it bit for bit with
 * the scalar expressions it pairs, compiled with the forward's flags.  mismatches (host, 8
 * entries) receives the count of differing values per piece: longwave recurrence downward and
 * upward, band fractions, half-level temperatures, blackbody terms, shortwave band 1, band 2,
 * heating-rate scaling.  All zero is the contract the forward's results rest on.  Synchronous
 * on the current device's default stream. */
int spd_selftest_packed(int n, uint32_t seed, unsigned int* mismatches);

/* ----------------------------------------------------------------------------------------- */
/* Held-Suarez forcing: HeldSuarezPhysics.compute_tendencies                                 */
/*   (jcm/physics/held_suarez/held_suarez_physics.py:76-101), the reference's second physics */
/* package, per element: Newtonian relaxation of T towards the radiative-equilibrium          */
/* temperature (equilibrium_temperature, :53-62; kt, :70-74) and Rayleigh drag on u and v     */
/* below sigma_b (kv, :64-68); the humidity tendency is zero.  Units are the caller's: rates   */
/* in 1/s and temperatures in K give tendencies in K/s and m/s^2 (the reference passes them    */
/* nondimensionalized by dinosaur's scales; the arithmetic is the same).                     */
/* ----------------------------------------------------------------------------------------- */
typedef struct {
  int32_t kx, ix, il, reserved;
  float sigma_b;          /* boundary-layer top (sigma) */
  float kf, ka, ks;       /* friction, free-atmosphere and surface relaxation rates */
  float min_t, max_t;     /* bounds of the equilibrium temperature */
  float dt_y, dthz;       /* its horizontal and vertical variations */
  float kappa;            /* R / cp */
  float sigma[SPD_MAX_KX];  /* level centres, top to bottom (coords.vertical.centers) */
} spd_hs_desc_t;

/* Latitude tables for spd_held_suarez: lat_tab[0][j] = sin(lat_j)^2, lat_tab[1][j] =
 * cos(lat_j)^2, lat_tab[2][j] = cos(lat_j)^4 (as the reference forms them), j < il, on the
 * device.  u, v, t are [kx][C] (C = ix*il), psa [C]; du, dv, dt, dq [kx][C], overlapping
 * neither the inputs nor one another (SPD_ERR_ALIAS). */
int spd_held_suarez(const spd_hs_desc_t* desc, const float* lat_tab, const float* u,
                    const float* v, const float* t, const float* psa, float* du, float* dv,
                    float* dt, float* dq, void* stream);

/* ----------------------------------------------------------------------------------------- */
/* Adjoint (vector-Jacobian product) of the plain forward.                                    */
/* Replaces jax.vjp of SpeedyPhysics.compute_tendencies (speedy_physics.py:88-127; the         */
/* reference differentiates through jax.checkpoint-ed terms, speedy_physics.py:82-86).         */
/* One thread per column re-evaluates the column's forward (nothing is kept from the forward  */
/* call) and runs a hand-written reverse pass over its terms.  Ties of min/max split the      */
/* derivative 0.5/0.5 (JAX's lax.min/lax.max rule); integer levels and the instance level set */
/* carry no derivative.  With SPD_FUSE_VERIFY set the VJP is that of the fused step           */
/* (verify_state, the physics, verify_tendencies and the humidity scale), and the humidity   */
/* gradient is with respect to the humidity as given.  `scratch` holds a one-member plan (the  */
/* instance's tile list, level-set word and per-latitude solar table), so that a single       */
/* instance runs the batched adjoint's kernels: spd_vjp_scratch_bytes(desc) bytes, 256-byte   */
/* aligned.                                                                                   */
/* ----------------------------------------------------------------------------------------- */
#define SPD_NUM_DIFF_PARAMS 12

/* Cotangents of the four tendency planes [kx][C]. */
typedef struct {
  const float *u_wind, *v_wind, *temperature, *specific_humidity;
} spd_cotangents_t;

/* Gradients with respect to the PhysicsState planes [kx][C] (u_wind and v_wind are nonzero only
 * at the lowest level, the only level the physics reads), psa [C], and the 12 differentiated
 * parameters in the order psmin, trcnv, rhil, rhbl, entmax, smf, trlsc, rhlsc, drhlsc, rhblsc,
 * albcl, albcls (params.py:11-16, :51-54, :72-73), summed over columns. */
typedef struct {
  float *u_wind, *v_wind, *temperature, *specific_humidity, *geopotential;
  float *normalized_surface_pressure;
  float *params;
} spd_grads_t;

size_t spd_vjp_scratch_bytes(const spd_desc_t* desc);

int spd_vjp(const spd_desc_t* desc, const spd_vgrid_t* vgrid, const spd_params_t* params,
            const spd_inputs_t* in, const spd_cotangents_t* ct, const spd_grads_t* grads,
            void* scratch, size_t scratch_bytes, void* stream);

/* ----------------------------------------------------------------------------------------- */
/* Batched ragged ensemble: many instances ("members") of mixed resolution and level count,  */
/* e.g. a forecast ensemble or a set of independent grids, in one fused launch over every      */
/* member's columns (and a fixup launch that redoes the members whose predicted level set       */
/* missed, or a level-set launch first under SPD_NO_SPECULATION).  Each                        */
/* member gives the same results as spd_fwd on it alone.  There is no reference counterpart   */
/* for the batching itself; per member it replaces SpeedyPhysics.compute_tendencies           */
/* (speedy_physics.py:88-127).                                                               */
/* ----------------------------------------------------------------------------------------- */
#define SPD_MAX_CLASSES 4

/* What the members of one class share: level count, switches, date (desc; desc.ix/il are
 * ignored), vertical grid and parameters. */
typedef struct {
  spd_desc_t desc;
  spd_vgrid_t vgrid;
  spd_params_t params;
} spd_class_t;

/* One member: its fields (device pointers, spd_fwd layout), shape and class index. */
typedef struct {
  spd_inputs_t in;
  spd_outputs_t out;
  int32_t ix, il, cls, reserved;
} spd_member_t;

/* Host-side summary of a plan, returned by spd_ensemble_plan and passed to spd_ensemble_fwd. */
typedef struct {
  int32_t nmembers, ntiles;
  uint64_t levelset_offset, levelset_bytes; /* the per-member level-set words (zeroed per call) */
  uint64_t plan_bytes;
} spd_plan_info_t;

/* Bytes of the device plan for these members (member table, tile list, level-set words,
 * per-member solar tables). */
size_t spd_ensemble_plan_bytes(const spd_member_t* members, int nmembers);

/* Builds the plan in host memory `plan_host` (plan_bytes long) for a device buffer at
 * `plan_device` (256-byte aligned); the caller copies plan_host to plan_device once, and may
 * reuse it for every call while the members' buffers stay where they are. */
int spd_ensemble_plan(const spd_class_t* classes, int nclasses, const spd_member_t* members,
                      int nmembers, void* plan_host, void* plan_device, size_t plan_bytes,
                      spd_plan_info_t* info);

/* Runs every member.  grid_blocks = 0 picks SMs x resident blocks for both launches (each
 * block strides over the tile list: the fastest form on an otherwise idle GPU); a positive
 * value sets the second launch's persistent grid (the autotuner's knob); SPD_GRID_PER_TILE
 * launches one block per tile for both launches, which shares the GPU better with concurrent
 * kernels (a late-starting persistent block still owns its whole stride of tiles). */
#define SPD_GRID_PER_TILE (-1)
int spd_ensemble_fwd(const spd_class_t* classes, int nclasses, void* plan_device,
                     const spd_plan_info_t* info, int grid_blocks, void* stream);

/* Timing hook (no reference counterpart): spd_ensemble_fwd, recording `event` (a cudaEvent_t,
 * or NULL) on `stream` between its two launches (see spd_fwd_marked), which then run in plain
 * stream order. */
int spd_ensemble_fwd_marked(const spd_class_t* classes, int nclasses, void* plan_device,
                            const spd_plan_info_t* info, int grid_blocks, void* stream,
                            void* event);

/* Batched adjoint: the VJP of every member of a ragged ensemble in one pre-pass launch and one
 * adjoint launch (no reference counterpart for the batching; per member it is spd_vjp).  Each
 * member gives the same gradients as spd_vjp on it alone; its 12 parameter gradients are its
 * own (grads.params of each member, zeroed by the call). */
typedef struct {
  spd_inputs_t in;
  spd_cotangents_t ct;
  spd_grads_t grads;
  int32_t ix, il, cls, reserved;
} spd_vjp_member_t;

size_t spd_ensemble_vjp_plan_bytes(const spd_vjp_member_t* members, int nmembers);

int spd_ensemble_vjp_plan(const spd_class_t* classes, int nclasses,
                          const spd_vjp_member_t* members, int nmembers, void* plan_host,
                          void* plan_device, size_t plan_bytes, spd_plan_info_t* info);

/* grid_blocks = 0: one block per tile (short blocks, so the SMs turn over and kernels of a
 * higher-priority stream get them quickly); otherwise a persistent grid of that many blocks. */
int spd_ensemble_vjp(const spd_class_t* classes, int nclasses, void* plan_device,
                     const spd_plan_info_t* info, int grid_blocks, void* stream);

/* ----------------------------------------------------------------------------------------- */
/* No-allocation variant of spd_fwd.  It has no counterpart in the reference.                 */
/*                                                                                            */
/* For callers that cannot allocate device memory or pass a scratch buffer through their      */
/* binding: a foreign-function bridge that only forwards the state, forcing and tendency      */
/* buffers it was given, or a process whose device memory belongs to another runtime's        */
/* pooling allocator.  Same computation and results as spd_fwd, but no scratch argument and   */
/* no allocation: the scratch lives in a fixed device array of the library (65,792 bytes on   */
/* every GPU that loads it, kept until process exit), which limits instances to                */
/* il <= SPD_NOALLOC_MAX_IL latitudes (SPD_ERR_NOALLOC_LIMIT otherwise).                      */
/*  - Every call looks up the array's device address in the current device's context          */
/*    (cudaGetSymbolAddress), so the address never outlives its context (cudaDeviceReset      */
/*    included).  The first call on a device also loads the library's kernels there; make     */
/*    that first call before any stream capture.                                              */
/*  - The stream must belong to the current device (SPD_ERR_STREAM_DEVICE otherwise): the     */
/*    array used is the current device's.                                                     */
/*  - Every call uses the same array and clears its level-set word itself.  Calls whose work   */
/*    overlaps on the GPU (other streams, other host threads) race on the array and corrupt    */
/*    each other's results: order them, for example on one stream.                            */
/* ----------------------------------------------------------------------------------------- */
#define SPD_NOALLOC_MAX_IL 2048
int spd_fwd_noalloc(const spd_desc_t* desc, const spd_vgrid_t* vgrid, const spd_params_t* params,
                    const spd_inputs_t* in, const spd_outputs_t* out, void* stream);

/* ----------------------------------------------------------------------------------------- */
/* Helpers                                                                                    */
/* ----------------------------------------------------------------------------------------- */
const char* spd_status_string(int status);
int spd_abi_version(void);
/* Fills `params` with Parameters.default() (params.py:244-254). */
void spd_default_params(spd_params_t* params);

#ifdef __cplusplus
}
#endif
#endif /* SPEEDY_B200_H */
