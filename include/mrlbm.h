/*
 * mrlbm.h -- C ABI of the B200 moment-representation LBM (MR-LBM) library.
 *
 * The reference solver (CERNN/MR-LBM) has no runtime plugin interface: its
 * boundary is a compile-time case API, one fused kernel launched from main(),
 * and its on-disk formats.  Each entry point below names the reference
 * interface it replaces (paths relative to the reference's source tree).
 *
 * Conventions
 *   - Every function returns an mrlbm_status; 0 is success.  Nothing calls
 *     exit(); the message of the last failure on the calling thread is
 *     available from mrlbm_last_error().
 *   - Host buffers are owned by the caller.  Device memory is owned by the
 *     handle that allocated it.
 *   - A handle is thread-compatible, not thread-safe: one host thread at a time.
 *   - "x-fastest" arrays are indexed x + nx*(y + ny*z) (the reference's
 *     idxScalarGlobal, src/globalFunctions.h:271-275).
 *   - "reference layout" is the reference's block-interleaved moment array
 *     idxMom (src/globalFunctions.h:31-42) with 8x8x8 blocks; it needs nx, ny
 *     and nz to be multiples of 8, like the reference.
 *   - Stored moments use the reference's scaled form (src/arrayIndex.h:8-17,
 *     186-187): rho-rho0, 3u, 4.5*Pi_xx, 9*Pi_xy, 9*Pi_xz, 4.5*Pi_yy, 9*Pi_yz,
 *     4.5*Pi_zz (+ omega as moment 10 when the viscosity is non-Newtonian;
 *     + C, 3 sum g c_x, 3 sum g c_y, 3 sum g c_z as moments 10-13 with the
 *     thermal scalar).
 */
#ifndef MRLBM_H
#define MRLBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MRLBM_OK = 0,
    MRLBM_EINVAL = 1,     /* bad argument or unsupported configuration */
    MRLBM_ENOMEM = 2,     /* device or host allocation failed / over budget */
    MRLBM_ECUDA = 3,      /* a CUDA call failed */
    MRLBM_EIO = 4,        /* file could not be read or written */
    MRLBM_EDIVERGED = 5,  /* NaN/Inf or |u| above the stability limit */
    MRLBM_ETIMEDOUT = 6,  /* a bounded device wait gave up */
    MRLBM_ENOTFOUND = 7,  /* unknown request / handle */
    MRLBM_EBUSY = 8,      /* no free slot / request still queued or running */
    MRLBM_ECANCELED = 9,  /* request cancelled */
    MRLBM_EBOUNDS = 10    /* bounds-check build: a step kernel skipped an out-of-range access */
} mrlbm_status;

typedef enum { MRLBM_D3Q19 = 19, MRLBM_D3Q27 = 27 } mrlbm_lattice;
/* Stored precision of the moments (arithmetic is FP32 in every case).
 * MRLBM_F16U ("split velocity"): rho - rho0 and the second moments in fp16,
 * each component of 3u in two fp16 words (the high word and what it rounds
 * away), 26 bytes a node instead of 20 (fp16) or 40 (fp32): velocity keeps
 * about 22 significant bits, which plain 16-bit storage loses step by step
 * at low viscosity.  Not with the thermal scalar or outflow walls.  No
 * reference counterpart (its dfloat is float or double, src/var.h:13-21). */
typedef enum { MRLBM_F32 = 0, MRLBM_F16 = 1, MRLBM_BF16 = 2, MRLBM_F16U = 3 } mrlbm_storage;
typedef enum { MRLBM_NEWTONIAN = 0, MRLBM_POWERLAW = 1, MRLBM_BINGHAM = 2 } mrlbm_rheology;

/* Node-type words follow the reference's nodeTypeMap (src/nodeTypeMap.h:10-80):
 * bits 0-7 octant solid mask (0 = bulk, 0xFF = solid), bits 8-10 BC kind
 * (0 no-slip wall, 1 prescribed-velocity wall, 2 outflow: a face node takes
 * its inward neighbour's previous-step moments, as the reference's
 * mountedCube / externalFlow cases do), bits 11-12 velocity index. */
#define MRLBM_NODE_BULK 0x00u
#define MRLBM_NODE_SOLID 0xFFu
/* a voxel's neighbour whose type is still to be derived (the reference's
 * MISSING_DEFINITION, src/nodeTypeMap.h) */
#define MRLBM_NODE_UNRESOLVED 0xFFFFFFFFu
#define MRLBM_BC_VELOCITY_WALL (1u << 8)
#define MRLBM_BC_OUTFLOW (2u << 8)
#define MRLBM_BC_VELOCITY_INDEX(k) (((uint32_t)(k) & 3u) << 11)
/* Thermal rule of a boundary node (bits 13-14) and its wall value index into
 * mrlbm_desc.t_wall (bits 15-16): the per-case g_bc_definition.inc switch of
 * the reference, as run-time data.  Bulk nodes always take C = sum g + source.
 *   0  C and its flux keep their stored values (node types the case's
 *      g_bc_definition.inc does not list)
 *   1  C = t_wall, flux 0 (src/cases/thermal_2D/g_bc_definition.inc)
 *   2  C = t_wall, flux along the wall normal copied from the inward
 *      neighbour's previous-step value, tangential flux 0
 *      (src/cases/rayleighBenard_Periodic/g_bc_definition.inc EAST/WEST)
 *   3  adiabatic: populations arriving from the solid side mirrored across the
 *      wall plane, C and flux from the sums
 *      (src/cases/rayleighBenard_Closed/g_bc_definition.inc NORTH/SOUTH)
 * Rules 2 and 3 need a face node (one solid half of the octant mask). */
#define MRLBM_THERMAL_KEEP 0u
#define MRLBM_THERMAL_DIRICHLET 1u
#define MRLBM_THERMAL_DIRICHLET_FLUX 2u
#define MRLBM_THERMAL_ADIABATIC 3u
#define MRLBM_THERMAL_RULE(r) (((uint32_t)(r) & 3u) << 13)
#define MRLBM_THERMAL_INDEX(k) (((uint32_t)(k) & 3u) << 15)

/* Run-time description of one domain: the physics that a reference case fixes
 * at compile time in constants.inc / model.inc (src/cases/<case>/). */
typedef struct {
    int nx, ny, nz;
    int lattice;            /* MRLBM_D3Q19 or MRLBM_D3Q27 (model.inc D3Qxx) */
    int storage;            /* mrlbm_storage: precision of the stored moments */
    int periodic[3];        /* 1 = BC_<axis>_PERIODIC, 0 = BC_<axis>_WALL */
    double tau;             /* relaxation time (constants.inc TAU) */
    double rho0;            /* RHO_0 */
    double force[3];        /* body force FX, FY, FZ (lattice units) */
    double bc_velocity[4][3]; /* wall velocity per velocity index (UX_BC..UZ_BC) */
    int rheology;           /* mrlbm_rheology (model.inc POWERLAW / BINGHAM) */
    double nnf_n;           /* power-law index N_INDEX */
    double nnf_k;           /* power-law consistency K_CONSISTENCY (0: rho0*(tau-1/2)/3) */
    double nnf_yield;       /* Bingham yield stress S_Y */
    double nnf_omega_p;     /* Bingham plastic omega OMEGA_P (0: 1/tau) */
    int bc_matrix_q;        /* 0: reference behaviour (19 on D3Q27, i.e. the
                               D3Q19 wall closed forms), or 19 / 27 explicitly */
    /* Thermal scalar C transported on D3G19 (constants.inc THERMAL_MODEL:
     * SECOND_DIST + CONVECTION_DIFFUSION_TRANSPORT, src/mlbm.cu:157-191,
     * 515-522, 603-616).  Four more stored moments follow the flow's: C and
     * 3 sum g c (M2_C_INDEX, M2_CX..CZ_INDEX, src/arrayIndex.h:42-50).
     * Supported on D3Q19, FP32 storage, Newtonian flow. */
    int thermal;            /* 1: transport C */
    double t_diffusivity;   /* T_DIFFUSIVITY (alpha); the relaxation uses the reference's
                               G_DIFF_FLUC_COEF with T_DIFF_REF = 1/6 */
    double t_reference;     /* T_REFERENCE: Boussinesq reference, initial and exterior C */
    double t_gravity_beta[3]; /* gravity_vector * T_gravity_t_beta: bulk nodes get the force
                               t_gravity_beta * rho0 * (C - t_reference) */
    double t_source;        /* T_Q_INTERNAL_D_Cp, added to C at bulk nodes every step */
    double t_wall[4];       /* wall temperatures by thermal value index (T_HOT, T_COLD, ...) */
    int reserved[8];
} mrlbm_desc;

typedef struct mrlbm_domain mrlbm_domain;

/* FP64 global sums over non-solid nodes (the reference's FP32 reductions,
 * src/reduction.cu:100-155, done in double). */
typedef struct {
    double mass;            /* sum rho */
    double momentum[3];     /* sum rho u */
    double kinetic_energy;  /* sum rho |u|^2 / 2 */
    double fluid_nodes;
    double max_speed;       /* max |u| */
    double nonfinite;       /* count of non-finite moments */
} mrlbm_sums;

const char* mrlbm_last_error(void);
const char* mrlbm_version(void);

/* Device selection for the calling host thread (the reference hard-codes
 * GPU_INDEX, src/var.h:31) and pinned host buffers for fast transfers. */
mrlbm_status mrlbm_set_device(int device);
mrlbm_status mrlbm_device_count(int* count);
mrlbm_status mrlbm_host_alloc(size_t bytes, void** ptr);
mrlbm_status mrlbm_host_free(void* ptr);

/* Allocation + setup.  Replaces allocateDeviceMemory/interfaceMalloc
 * (src/main.cuh:455-900) for one case. */
mrlbm_status mrlbm_domain_create(const mrlbm_desc* desc, mrlbm_domain** out);
mrlbm_status mrlbm_domain_destroy(mrlbm_domain* dom);
/* Device bytes held by a domain of this description (moments, node classes). */
mrlbm_status mrlbm_domain_bytes(const mrlbm_desc* desc, size_t* bytes);

/* Node types, x-fastest, reference nodeTypeMap words.  Replaces
 * hostInitialization_nodeType / bc_initialization.inc
 * (src/lbmInitialization.cu:958-975). */
mrlbm_status mrlbm_set_node_types(mrlbm_domain* dom, const uint32_t* node_type);
/* Case mode: node types whose boundary nodes are handled by a case's own
 * compiled bc_definition.inc (mr-lbm_b200/casebuild.py); any word is accepted
 * and handed to the snippet unchanged (the reference's kernel switch,
 * src/mlbm.cu:457-461).  Only step kernels built by casebuild.py can step
 * such a domain. */
mrlbm_status mrlbm_set_node_types_case(mrlbm_domain* dom, const uint32_t* node_type);

/* Initial state from physical rho, u fields (x-fastest, host).  Replaces
 * gpuInitialization_mom + flow_initialization.inc
 * (src/lbmInitialization.cu:28-131), including its D3Q19-sum second moments. */
mrlbm_status mrlbm_init_flow(mrlbm_domain* dom, const float* rho, const float* ux, const float* uy,
                             const float* uz);
/* Built-in initial states computed on the device:
 * uniform rho0 and velocity (u0[3]), and the Taylor-Green vortex of
 * src/cases/taylorGreen/flow_initialization.inc:1-4 with amplitude u0 and
 * length scale L (L = N / 2pi in the reference). */
mrlbm_status mrlbm_init_uniform(mrlbm_domain* dom, const double u0[3]);
mrlbm_status mrlbm_init_taylor_green(mrlbm_domain* dom, double u0, double L);

/* Advance nsteps fused collide-stream steps on the domain's stream.  Replaces
 * the gpuMomCollisionStream launch + swapGhostInterfaces loop
 * (src/main.cu:200-230, src/mlbm.cu:3-714); no host sync per step. */
mrlbm_status mrlbm_step(mrlbm_domain* dom, int nsteps);
/* Same, recorded once into a CUDA graph and replayed (for small domains where
 * launch cost matters). */
mrlbm_status mrlbm_step_graph(mrlbm_domain* dom, int nsteps);
/* Device-timed nsteps: CUDA events on the domain's stream around the launches. */
mrlbm_status mrlbm_time_steps(mrlbm_domain* dom, int nsteps, float* ms);
mrlbm_status mrlbm_synchronize(mrlbm_domain* dom);
/* Self-test of the bounded device waits that guard every tile load of the
 * step kernels (no counterpart in the reference, whose kernel has none): a
 * one-CTA kernel waits on a barrier that is never completed, gives up after
 * `polls` polls (1..2^26; the step kernels use 2^26), raises the device error
 * flag and exits.  Returns MRLBM_ETIMEDOUT (the expected outcome) with the
 * kernel's duration in *seconds; the context stays usable. */
mrlbm_status mrlbm_selftest_bounded_wait(unsigned polls, double* seconds);
mrlbm_status mrlbm_get_step(mrlbm_domain* dom, int* step);
/* z planes each CTA of the single-domain step marches (0: chosen from the
 * grid so the last wave of CTAs is full; otherwise 1..nz).  A tuning knob with
 * no effect on results: every chunk gives bit-identical moments.  The
 * reference's counterpart is its fixed 8^3 block (src/definitions.h:87-92). */
mrlbm_status mrlbm_set_z_chunk(mrlbm_domain* dom, int lz);
mrlbm_status mrlbm_get_z_chunk(mrlbm_domain* dom, int* lz);

/* Tile-ordered steps (on = 1, the default): within one mrlbm_step call each
 * step launch may start while the one before it finishes, and a tile waits
 * only for the previous step's tiles around it (a per-tile word on the
 * device, with a bounded wait that raises MRLBM_ETIMEDOUT), so the SMs that
 * the last CTAs of a step leave idle already run the next step.  on = 0
 * orders whole launches.  Results are bit-identical either way.  Domains
 * with outflow walls or a thermal scalar always order whole launches.  No
 * reference counterpart (one kernel launch per step, src/main.cu:183-200). */
mrlbm_status mrlbm_set_tile_order(mrlbm_domain* dom, int on);

/* Launch on a caller's stream (a cudaStream_t of the domain's device; NULL
 * returns to the domain's own stream, so the legacy default stream cannot be
 * chosen).  The stream must outlive the domain or be reset first.  Work already queued on the previous
 * stream is ordered before anything queued afterwards.  No reference
 * counterpart (the reference launches on the default stream, src/main.cu:183). */
mrlbm_status mrlbm_set_stream(mrlbm_domain* dom, void* stream);
mrlbm_status mrlbm_get_stream(mrlbm_domain* dom, void** stream);

/* Z-slab decomposition: one domain cut into slabs of whole z planes, each an
 * ordinary domain (non-periodic in z) on its own GPU or all on one.  After
 * every step each slab's z ghost planes are filled from its neighbours'
 * boundary planes; the step kernel then reads them locally.  The reference is
 * single-GPU (README.md:38); the exchanged planes play the part of its Z_0 /
 * Z_1 ghost faces (src/globalStructs.h ghostInterfaceData, the z faces).
 *
 * A plane is, for every moment pair, one padded z plane of the buffer the next
 * step reads (x/y ghost shell included, so periodic x/y copies travel with
 * it): npairs blocks of `bytes` bytes, `pair_stride` bytes apart, starting at
 * device address `base`.  The pointers change after every step (ping-pong). */
#define MRLBM_ZPLANE_FIRST 0        /* interior plane z = 0: goes to the slab below */
#define MRLBM_ZPLANE_LAST 1         /* interior plane z = nz - 1: goes to the slab above */
#define MRLBM_ZGHOST_BELOW 2        /* ghost plane z = -1: filled from the slab below */
#define MRLBM_ZGHOST_ABOVE 3        /* ghost plane z = nz: filled from the slab above */
typedef struct {
    void* base;
    long long pair_stride;
    long long bytes;
    int npairs;
    int device;
} mrlbm_zplane;
mrlbm_status mrlbm_zslab_plane(mrlbm_domain* dom, int which, mrlbm_zplane* out);
/* Device copy of src's plane `src_which` (FIRST or LAST) into dst's ghost plane
 * `dst_which` (BELOW or ABOVE): one strided copy on src's stream, ordered after
 * the work queued on both domains' streams and before dst's later work.  The
 * two domains must have the same nx, ny, lattice, storage and moments. */
mrlbm_status mrlbm_zslab_copy(mrlbm_domain* src, int src_which, mrlbm_domain* dst, int dst_which);
/* The exchange across processes (one slab per rank), for C/C++ callers: NCCL
 * point-to-point operations of all moment pairs' planes, in place, in one NCCL
 * group queued on the domain's stream after its steps (no host wait).  The
 * library opens libnccl.so.2 itself.  mrlbm_nccl_unique_id writes a
 * 128-byte id that the caller hands to every rank (its own transport);
 * mrlbm_nccl_comm_init makes this rank's communicator on the current device;
 * rank_below / rank_above are the ranks of the neighbouring slabs in that
 * communicator, -1 at a non-periodic end, the own rank for a single periodic
 * slab.  Every rank lists the upward plane before the downward one, so sends
 * and receives pair up in NCCL's per-peer order.  No reference counterpart
 * (the reference is single-GPU, README.md:38). */
mrlbm_status mrlbm_nccl_unique_id(void* id);
mrlbm_status mrlbm_nccl_comm_init(int nranks, const void* id, int rank, void** comm);
mrlbm_status mrlbm_nccl_comm_destroy(void* comm);
mrlbm_status mrlbm_zslab_exchange_nccl(mrlbm_domain* dom, void* comm, int rank_below, int rank_above);

/* Moments in the reference's idxMom layout (fMom, host float buffer of
 * nx*ny*nz*num_moments).  Used by checkpoints and drop-in callers. */
mrlbm_status mrlbm_num_moments(mrlbm_domain* dom, int* nm);
mrlbm_status mrlbm_get_moments_ref_layout(mrlbm_domain* dom, float* fmom);
mrlbm_status mrlbm_set_moments_ref_layout(mrlbm_domain* dom, const float* fmom);
/* Moments as float, [moment][z][y][x] (x fastest). */
mrlbm_status mrlbm_get_moments(mrlbm_domain* dom, float* m);
mrlbm_status mrlbm_set_moments(mrlbm_domain* dom, const float* m);
/* Macroscopic fields as saveMacr writes them (src/saveData.cu:62-74):
 * rho = rho0 + m0, u = stored 3u (NOT divided by 3), x-fastest.  Any pointer
 * may be NULL. */
mrlbm_status mrlbm_get_macr(mrlbm_domain* dom, float* rho, float* ux, float* uy, float* uz, float* omega);

/* FP64 reductions (mass, momentum, kinetic energy, divergence watch).  Replaces
 * sumReductionThread_* + sumReductionBlock + totalKineticEnergy
 * (src/reduction.cu:37-243, src/treatData.cu:105-165). */
mrlbm_status mrlbm_reduce_fp64(mrlbm_domain* dom, mrlbm_sums* out);
/* Steady-state residual ||u^n - u^ref||_2 / (||u^n||_2 + 1e-30) over fluid
 * nodes, FP64, against the snapshot taken by the previous call (the first
 * call takes the snapshot and returns 1). */
mrlbm_status mrlbm_residual(mrlbm_domain* dom, double* residual);

/* The sums of mrlbm_reduce_fp64 (every node counted: the field carries no node
 * types) for a caller-owned FP32 field in the reference's idxMom layout
 * (fmom: device memory of the current device, nx*ny*nz*num_moments floats,
 * nx, ny, nz multiples of 8; stream may be NULL), computed without allocating
 * anything.  No counterpart in the reference: its reductions of fMom
 * (src/auxFunctions.cu:8-58, src/treatData.cu:105-165) cudaMalloc a partials
 * buffer on every call.
 * Scratch: a file-scope __device__ array of 37,952 bytes per device (592 block
 * partials + 8 results); the call always uses 592 blocks and strides over
 * larger fields, so every field size fits it.  Nothing in it has to start at
 * zero (each call writes what it reads).  The first call in each CUDA context
 * of a device looks up the array's address (cudaGetSymbolAddress, with that
 * device current).  Every call synchronises `stream` to return the sums on
 * the host, so no call can be made while `stream` is being captured.  Calls
 * share the array per device, so calls whose executions overlap on one device
 * (two host threads, or unordered streams) race and return wrong sums:
 * serialise them.  fmom may also be managed memory.  For a field with the same
 * values as a domain's F32 moments the result equals mrlbm_reduce_fp64's for
 * that domain (same blocks, same summation order). */
mrlbm_status mrlbm_reduce_fp64_ref_layout_noalloc(const float* fmom, int nx, int ny, int nz, int num_moments,
                                                  double rho0, void* stream, mrlbm_sums* out);

/* Files in the reference formats. */
/* <path>/<id>/checkpoint/_curr_step.bin, _fMom.bin, _fGhost.{X,Y,Z}_{0,1}.bin
 * (src/checkpoint.cu:129-186, 372-382; POSIX separators). */
mrlbm_status mrlbm_save_checkpoint(mrlbm_domain* dom, const char* path_files, const char* id_sim, int step);
/* Loads the same file set; *step receives the saved step + 1 (checkpoint.cu:157-159). */
mrlbm_status mrlbm_load_checkpoint(mrlbm_domain* dom, const char* path_files, const char* id_sim, int* step);
/* <path>/<id>/<id>_{rho,ux,uy,uz[,omega]}NNNNNN.bin (src/saveData.cu:62-260, 439-467). */
mrlbm_status mrlbm_save_macr_bin(mrlbm_domain* dom, const char* path_files, const char* id_sim, int step);
/* Legacy VTK structured points, binary big-endian, as saveVarVTK writes it
 * (src/saveData.cu:303-400): rho, velocity (physical u), omega when present;
 * <path>/<id>/<id>_vtk<step>.vtk (src/saveData.cu:153). */
mrlbm_status mrlbm_save_vtk(mrlbm_domain* dom, const char* path_files, const char* id_sim, int step);
/* <path>/<id>/<id>_info.txt (src/saveData.cu:469-613); case_name = BC type. */
mrlbm_status mrlbm_save_info(mrlbm_domain* dom, const char* path_files, const char* id_sim,
                             const char* case_name, int nsteps, double mlups);
/* The same text for a description alone, on the host (no device work; BY and
 * BZ are the step geometry of the description without wall classes on a
 * 148-SM B200): *len receives its length; buf (may be NULL to query) must hold
 * len + 1 bytes. */
mrlbm_status mrlbm_info_text(const mrlbm_desc* desc, const char* id_sim, const char* case_name, int nsteps,
                             double mlups, char* buf, size_t cap, size_t* len);

/* ------------------------------------------------------------------ batches
 * Many independent domains of uneven sizes advanced together by one
 * persistent kernel per step: every domain's (x, y) columns and z chunks form
 * one work list; persistent CTAs take work items from a device-side ticket
 * counter; the step launches are captured once in a CUDA graph and replayed.
 * The reference runs one domain per process (src/main.cu); this has no
 * counterpart there.  All domains of a batch share the lattice and the storage
 * precision; the supported physics per domain are periodic/no-BC, walls and
 * velocity walls (with or without body force), and power-law walls with body
 * force (the serving mix).  Domain ids stay valid until removed. */
typedef struct mrlbm_batch mrlbm_batch;

mrlbm_status mrlbm_batch_create(int lattice, int storage, mrlbm_batch** out);
mrlbm_status mrlbm_batch_destroy(mrlbm_batch* batch);
/* Adds a domain (allocates its moment buffers); *id receives its handle. */
mrlbm_status mrlbm_batch_add(mrlbm_batch* batch, const mrlbm_desc* desc, int* id);
mrlbm_status mrlbm_batch_remove(mrlbm_batch* batch, int id);
/* The domain object of a member, for set-up and read-back with the
 * single-domain calls above (node types, init, moments, reductions, files).
 * Do not step it directly while it belongs to the batch. */
mrlbm_status mrlbm_batch_domain(mrlbm_batch* batch, int id, mrlbm_domain** dom);
/* Advance every member by nsteps (graph replay; eager launches for a short
 * remainder). */
mrlbm_status mrlbm_batch_step(mrlbm_batch* batch, int nsteps);
mrlbm_status mrlbm_batch_synchronize(mrlbm_batch* batch);
/* Device-timed nsteps of the whole batch (CUDA events around the launches). */
mrlbm_status mrlbm_batch_time_steps(mrlbm_batch* batch, int nsteps, float* ms);
/* Work items (columns) in the current list, lattice nodes of all members. */
mrlbm_status mrlbm_batch_info(mrlbm_batch* batch, int* members, int* items, long long* nodes);
/* Autotuner, for each of the kernel's two tile heights (8 rows, two CTAs an
 * SM; 14 rows, one): measures the z-chunk length per domain-size class (a few
 * timed steps of the whole batch per candidate), then times the batch with
 * those chunks; keeps the faster height (the starting one unless the other
 * is 2 % faster) and its chunks.  It times on the members themselves and
 * restores their moments and step counts afterwards.  Without it: 8 rows
 * (14 for D3Q27 split-velocity fp16 batches) and 32-plane chunks. */
mrlbm_status mrlbm_batch_autotune(mrlbm_batch* batch);
/* The batch kernel's tile height: 8 or 14 interior rows per CTA (results do
 * not depend on it; no counterpart in the reference). */
mrlbm_status mrlbm_batch_set_rows(mrlbm_batch* batch, int rows);
mrlbm_status mrlbm_batch_get_rows(mrlbm_batch* batch, int* rows);
/* The z-chunk length the batch uses for a domain of this size. */
mrlbm_status mrlbm_batch_chunk_for(mrlbm_batch* batch, int nx, int ny, int nz, int* lz);

/* ------------------------------------------------------------------ serving
 * A continuous-batching solve server (no counterpart in the reference, which
 * runs one case per process).  Requests queue in arrival order; a tick admits
 * queued requests while their device bytes fit the HBM budget and a slot is
 * free, advances every active solve by steps_per_tick steps in one batch,
 * then retires solves whose residual ||u^n - u^(n-k)|| / ||u^n|| (FP64, k =
 * steps_per_tick) is at most residual_tol, that reached max_steps, or that
 * diverged (NaN/Inf or |u| > 0.3: status MRLBM_EDIVERGED).  Times are seconds
 * on the server's monotonic clock; latency = retirement - arrival. */
typedef struct mrlbm_server mrlbm_server;

typedef enum { MRLBM_REQ_LID_CAVITY = 0, MRLBM_REQ_DUCT = 1 } mrlbm_request_kind;

typedef struct {
    int kind;               /* mrlbm_request_kind */
    int n;                  /* cubic edge length */
    double re;              /* cavity: Reynolds number (lid 0.05, tau from Re) */
    double lid_u;           /* cavity: lid velocity (0: 0.05) */
    double nnf_n;           /* duct: power-law index */
    double tau;             /* duct: tau of the consistency K = rho0 (tau - 1/2) / 3 (0: 0.8) */
    double force_z;         /* duct: body force along z (0: sized for u_max ~ 0.05) */
    double solid_fraction;  /* duct: Bernoulli obstacle fraction on interior nodes */
    uint64_t seed;          /* duct: obstacle mask seed */
    double arrival;         /* arrival time (seconds, server clock); < 0: now */
} mrlbm_request;

typedef struct {
    int status;             /* MRLBM_OK done, MRLBM_EBUSY queued/running, MRLBM_EDIVERGED, ... */
    int steps;
    double residual;
    double arrival, admitted, finished;  /* server clock, seconds */
} mrlbm_request_result;

typedef struct {
    int queued, active, done, failed;
    double hbm_in_use;      /* bytes */
    double p50_latency, p99_latency, mean_latency;  /* seconds, over finished solves */
    double solves_per_s;    /* finished solves / (last finish - first arrival) */
    double lattice_updates; /* total node updates done */
} mrlbm_server_stats;

mrlbm_status mrlbm_server_create(int storage, double hbm_budget_bytes, int max_active, int steps_per_tick,
                                 double residual_tol, int max_steps, mrlbm_server** out);
mrlbm_status mrlbm_server_destroy(mrlbm_server* srv);
/* Queue a request; *rid receives its id.  Requests that could never fit the
 * budget are refused with MRLBM_ENOMEM. */
mrlbm_status mrlbm_server_submit(mrlbm_server* srv, const mrlbm_request* req, int* rid);
mrlbm_status mrlbm_server_cancel(mrlbm_server* srv, int rid);
/* One scheduling tick (admit, step, retire).  *active receives the number of
 * running solves after the tick (0 and an empty queue: idle). */
mrlbm_status mrlbm_server_tick(mrlbm_server* srv, int* active);
mrlbm_status mrlbm_server_result(mrlbm_server* srv, int rid, mrlbm_request_result* out);
/* Final moments of a finished request (float [moment][z][y][x]); kept until
 * mrlbm_server_release. */
mrlbm_status mrlbm_server_moments(mrlbm_server* srv, int rid, float* m, size_t count);
mrlbm_status mrlbm_server_release(mrlbm_server* srv, int rid);
mrlbm_status mrlbm_server_stats_get(mrlbm_server* srv, mrlbm_server_stats* out);
mrlbm_status mrlbm_server_now(mrlbm_server* srv, double* t);
/* Test hook: replace one node's moments of an admitted request with NaN
 * (host-side fault injection; the divergence watch must retire it). */
mrlbm_status mrlbm_server_inject_nan(mrlbm_server* srv, int rid);
/* Compute limit of admission (0, the default: none).  A queued request
 * joins the running solves only while their lattice nodes together, its own
 * included, stay within `nodes`; with nothing running it always starts.
 * Admission stays in arrival order, so with a limit of about what fills the
 * GPU (a few million nodes on a B200) large solves run one or two at a time
 * in arrival order and small ones still share a batch: the same throughput
 * as sharing the GPU among every arrived request, and earlier completions
 * for the early arrivals.  No counterpart in the reference. */
mrlbm_status mrlbm_server_set_capacity(mrlbm_server* srv, double nodes);
/* Keep each finished request's final moments on the host for
 * mrlbm_server_moments (off by default: large requests are hundreds of MB). */
mrlbm_status mrlbm_server_keep_results(mrlbm_server* srv, int on);
/* A standalone domain for a request, set up exactly as the server sets up
 * its batch member (description, node types, initial state): for solving a
 * request alone with the single-domain calls. */
mrlbm_status mrlbm_request_domain(const mrlbm_request* req, int storage, mrlbm_domain** out);
/* What a request expands to, on the host only (no device work): its domain
 * description and, when node_types is not NULL, its n^3 node-type words
 * (x-fastest), as the server builds them.  No reference counterpart (a
 * reference case fixes both at compile time). */
mrlbm_status mrlbm_request_describe(const mrlbm_request* req, int storage, mrlbm_desc* desc, uint32_t* node_types);

/* Host-side node-type builders (no device work).
 * Voxel geometry: solid (x-fastest, nonzero = solid) -> nodeTypeMap words: solid
 * nodes 0xFF, fluid nodes the octant mask of their solid neighbours; neighbours
 * outside a non-periodic axis count as solid (domain walls).  Replaces bc_id +
 * define_voxel_bc (src/lbmInitialization.cu:1058-1227). */
mrlbm_status mrlbm_voxel_node_types(int nx, int ny, int nz, const uint8_t* solid, const int periodic[3],
                                    uint32_t* node_type);
/* Voxel files of the reference's obstacle cases (VOXEL_FILENAME, read by
 * read_xyz_file, src/lbmInitialization.cu:978-1039, called at src/main.cuh:
 * 996-1007): each "x,y,z" line marks that node MRLBM_NODE_SOLID and its 26
 * neighbours (axes wrapped periodically) MRLBM_NODE_UNRESOLVED unless solid;
 * lines outside the grid are skipped.  *voxels (may be NULL) receives the
 * count of solid lines read.  node_types is x-fastest. */
mrlbm_status mrlbm_voxel_mark_csv(const char* path, int nx, int ny, int nz, uint32_t* node_types, long long* voxels);
/* The reference's define_voxel_bc / bc_id (src/lbmInitialization.cu:1058-1227):
 * every MRLBM_NODE_UNRESOLVED node takes the octant mask of its solid
 * neighbours, axes wrapped periodically (all eight octants is 0xFF, solid). */
mrlbm_status mrlbm_voxel_resolve(int nx, int ny, int nz, uint32_t* node_types);
/* The lid-driven cavity typing of src/cases/lidDrivenCavity_3D/bc_initialization.inc:
 * the whole y = ny-1 face (edges and corners included) is the lid, a velocity
 * wall with the given velocity index; other boundary nodes are no-slip walls. */
mrlbm_status mrlbm_lid_cavity_node_types(int nx, int ny, int nz, int lid_velocity_index, uint32_t* node_type);
/* The moment-BC data the device uses for one node type (host only; for
 * inspection and tests).  out[0..48] A(omega0)^-1 row-major, out[49..55]
 * A^-1 e0, out[56..62] q^T A^-1, out[63] q^T A^-1 e0, out[64..66] wall
 * velocity; *known = bitmask of known populations. */
mrlbm_status mrlbm_bc_class_info(int lattice, int bc_matrix_q, uint32_t node_type, const double bc_velocity[4][3],
                                 double omega0, float* out, uint32_t* known);

#ifdef __cplusplus
}
#endif
#endif /* MRLBM_H */
