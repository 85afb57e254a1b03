/*
 * acp.h -- C ABI of the B200 engine for the acPulse_vcLBM hot path.
 *
 * The reference runs one process with a C++ object API: Control(file) reads
 * BoundaryConditions.txt (Control.cpp:8-132), Lattice(Control&) builds the
 * mesh (Lattice.h:23-57), initialization(Control&) sets the pulse
 * (Lattice.cpp:1397-1493) and solve(alt) / solve(alt0, alt1) advance one
 * coarse step (Lattice.cpp:2158-2210).  This header is the thin C layer that a
 * drop-in Control/Lattice (or a cgo / ctypes / JNI caller) binds: plain
 * structs, pointers and sizes, no C++ or torch types.  Every function returns
 * ACP_OK (0) or a negative ACP_ERR_* code; acp_last_error() gives the text.
 *
 * Units: the case descriptor is in the reference's SI units (metres, seconds,
 * kg/m^3).  Populations read back through acp_read_populations are the
 * reference's FP64 distributions f_i (Node::distr_, Node.h:190) of the array
 * the next step reads, i.e. post-streaming / pre-collision, for every storage
 * form.  Array order is structure-of-arrays: index ((q*nz + k)*ny + j)*nx + i.
 */
#ifndef ACP_H
#define ACP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ACP_ABI_VERSION 1

/* status codes */
#define ACP_OK 0
#define ACP_ERR_INVALID (-1)     /* bad argument or case description */
#define ACP_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define ACP_ERR_NOMEM (-3)       /* device or host allocation failed */
#define ACP_ERR_UNSUPPORTED (-4) /* valid but not built (e.g. option combination) */
#define ACP_ERR_NUMERIC (-5)     /* NaN/Inf or density blow-up detected on the device */
#define ACP_ERR_TIMEOUT (-6)     /* a bounded device wait gave up */
#define ACP_ERR_BUDGET (-7)      /* admission refused: HBM budget exhausted */
#define ACP_ERR_STATE (-8)       /* call out of order (e.g. step before init) */

/* Collision-Model keyword (BoundaryConditions.txt:30-44, Lattice.cpp:2158-2183) */
enum acp_op { ACP_OP_SRT = 0, ACP_OP_MRT_GS = 1, ACP_OP_MRT_RM = 2, ACP_OP_RR = 3, ACP_OP_HRR = 4 };

/* per-axis boundary: the reference puts LODI boundary nodes on all six faces
 * (Lattice.cpp:132,142); periodic axes are an extension used by the pulse
 * configurations (quasi-2D boxes periodic in y and z). */
enum acp_bc { ACP_BC_LODI = 0, ACP_BC_PERIODIC = 1 };

/* population storage form */
enum acp_storage {
    ACP_STORE_F64 = 0,     /* f_i as FP64 (the reference's representation) */
    ACP_STORE_F32_DEV = 1, /* f_i - w_i*rho0 as FP32, collided in FP32 */
    ACP_STORE_F16_DEV = 2  /* f_i - w_i*rho0 as FP16 with a power-of-two scale per population */
};

/* Coupling-Approach keyword (BoundaryConditions.txt:53) */
enum acp_coupling { ACP_COUPLING_STD = 0, ACP_COUPLING_DC1 = 1, ACP_COUPLING_DC2 = 2 };
/* F2C-Filter keyword (BoundaryConditions.txt:68) */
enum acp_f2c_filter { ACP_F2C_NOFI = 0, ACP_F2C_LAG = 1, ACP_F2C_TOU = 2 };
/* Scaling-Style keyword (BoundaryConditions.txt:89) */
enum acp_scaling { ACP_SCALING_SRT = 0, ACP_SCALING_MRT = 1 };
/* Coarse-to-Fine keyword (BoundaryConditions.txt:71-77) */
enum acp_c2f_replace { ACP_C2F_MF = 0, ACP_C2F_MFP = 1, ACP_C2F_FALL = 2 };
/* Fine-to-Coarse keyword (BoundaryConditions.txt:79-83) */
enum acp_f2c_replace { ACP_F2C_MC = 0, ACP_F2C_MCP = 1, ACP_F2C_CALL = 2 };

/* refinement layout */
enum acp_layout {
    ACP_LAYOUT_SHELL = 0, /* the reference's: fine shell around a coarse core (Lattice.cpp:17-234); the
                           * core spans [RefinementLayerX - Overlap, nx-1 - RefinementLayerYZ + Overlap]
                           * in x and [RefinementLayerYZ - Overlap, n-1 - RefinementLayerYZ + Overlap]
                           * in y and z; LODI on every face */
    ACP_LAYOUT_BOX = 1    /* fine box [box_lo, box_hi] (coarse node indices) inside the coarse grid */
};

/* initial condition */
enum acp_ic {
    ACP_IC_REFERENCE = 0, /* Lattice::initialization: Rc = 0.06 m, A = 0.01, centre -8 Rc in x (Lattice.cpp:1415-1433) */
    ACP_IC_GAUSSIAN = 1   /* rho = rho0 (1 + eps exp(-ln2 r^2 / b^2)), centre and b in coarse cells */
};

/* readable fields */
enum acp_field { ACP_FIELD_RHO = 0, ACP_FIELD_UX = 1, ACP_FIELD_UY = 2, ACP_FIELD_UZ = 3, ACP_FIELD_P = 4 };

typedef struct acp_case_desc {
    /* lattice (Control::getNumberOfNodes*, Control.cpp:43-45) */
    int nx, ny, nz;
    double spacing;            /* coarse spacing [m] (Spacing) */
    double domain_size[3];     /* Domain-Size-X/Y/Z [m]; the reference pulse is centred with them */
    /* physics (Density, KinematicViscosity, SpeedOfSound, MACH-Number) */
    double density, kinematic_viscosity, speed_of_sound, mach;
    /* collision */
    int op;                    /* enum acp_op */
    int eq_order;              /* Order-Of-Equilibrium: 2, 3 or 4 */
    int cubic_mach;            /* Cubic-Mach-Correction yes=1 (RR, HRR) */
    double hybrid_sigma;       /* Hybrid-Parameter (HRR) */
    int mrt_writeback;         /* 0: as the reference (collision result discarded, Node.cpp:2603,2833); 1: applied */
    /* boundaries */
    int bc[3];                 /* enum acp_bc per axis x, y, z */
    int transverse;            /* Transverse yes=1 */
    double k1;                 /* K1-Relaxation */
    /* refinement */
    int max_level;             /* MaxLevel: 0 or 1 */
    int layout;                /* enum acp_layout */
    int ref_layer_yz, ref_layer_x, overlap; /* RefinementLayerYZ, RefinementLayerX, Overlap (shell layout) */
    int box_lo[3], box_hi[3];  /* refined box in coarse node indices, inclusive (box layout) */
    int coupling;              /* enum acp_coupling */
    int f2c_filter;            /* enum acp_f2c_filter */
    int scaling_style;         /* enum acp_scaling */
    int c2f_replace;           /* enum acp_c2f_replace */
    int f2c_replace;           /* enum acp_f2c_replace */
    /* initial condition */
    int ic;                    /* enum acp_ic */
    double ic_eps, ic_b;       /* amplitude and half-width (coarse cells) for ACP_IC_GAUSSIAN */
    double ic_center[3];       /* centre in coarse node coordinates for ACP_IC_GAUSSIAN */
    int ic_dims;               /* 2: r^2 over x,y only (quasi-2D pulse); 3: over x,y,z */
    /* precision */
    int storage;               /* enum acp_storage */
    /* LODI relaxation length per axis in coarse nodes: the reference's L =
     * NumberOfNodes_axis * Spacing (Node.cpp:311); 0 takes the case's own
     * nx, ny, nz.  A slab of a lattice split in x keeps the whole lattice's. */
    int lodi_length_nodes[3];
    int reserved[5];
} acp_case_desc;

typedef struct acp_handle acp_handle;

/* Fill *d with the reference's defaults (BoundaryConditions.txt as shipped,
 * single level, FP64). */
void acp_default_case(acp_case_desc* d);

/* Parse a BoundaryConditions.txt file with the reference's keyword rules
 * (Control::readValue/readString, Control.cpp:135-204): first token matched
 * exactly, missing mandatory keyword is an error.  Optional keywords added by
 * this engine (Periodic-X/Y/Z, Pulse-*, Refinement-Box-*, Storage,
 * MRT-Write-Back, Layout) keep the reference defaults when absent. */
int acp_parse_case_file(const char* path, acp_case_desc* d, char* err, size_t err_len);

/* Replaces Lattice(Control&) (Lattice.h:23-57): validates the case, builds
 * the node types and boundary wiring, allocates device state.  device < 0
 * means the current device. */
int acp_create(const acp_case_desc* d, int device, acp_handle** out);
/* Replaces Lattice::initialization (Lattice.cpp:1397-1493). */
int acp_init(acp_handle* h);
/* Replaces n calls of Lattice::solve(alt) / solve(alt0, alt1)
 * (Lattice.cpp:2158-2210): n coarse steps, asynchronous on the handle's
 * stream. */
int acp_step(acp_handle* h, int n_coarse_steps);
/* Wait for the handle's stream; reports a device-side numeric fault. */
int acp_sync(acp_handle* h);
/* Node counts of a level's dense box (nodes = dims[0]*dims[1]*dims[2]). */
int acp_level_dims(acp_handle* h, int level, int dims[3]);
/* Level-global node index of a level's local node (0, 0, 0): the fine box's
 * corner (box layout) or the coarse core's corner (shell layout); level-global
 * indices of the fine level are twice the coarse ones. */
int acp_level_origin(acp_handle* h, int level, int origin[3]);
/* Nodes updated per coarse step, for MLUPS: coarse active + 2 * fine active. */
int acp_active_updates(acp_handle* h, long long* coarse_nodes, long long* fine_nodes);
/* Populations of a level as FP64 f_i (see header comment), host buffer of
 * 19 * nodes doubles; replaces Lattice::getDistribution (Lattice.h:119). */
int acp_read_populations(acp_handle* h, int level, double* host_out);
/* The level's other ping-pong array as FP64 f_i, same layout: what the
 * reference's getDistribution(flag, ...) returns for the flag that does not
 * name the current state (Lattice.h:119, Node.h:52).  The engine streams by
 * push from one array into the other, so this array holds the state the last
 * coarse step started from (coarse level; the fine level: its state at the
 * half step, after the coarse-to-fine coupling), where the reference keeps
 * the post-collision values of its in-place collision.  Before the first
 * step both arrays hold the initial state, as in the reference. */
int acp_read_populations_other(acp_handle* h, int level, double* host_out);
/* Kind of node (i, j, k) of a level (level-global node indices, as
 * getDistribution takes them) in the reference's node IDs: 0 FluidNode,
 * 1 BoundaryNode (LODI), 2 GridCoupling (FluidNode.h:11, BoundaryNode.h:11,
 * GridCoupling.h:12), or -1 where the level has no live node (covered by the
 * other level, or outside it).  *face_class: the face class
 * (fx+1)*9 + (fy+1)*3 + (fz+1) of a boundary node's domain faces or of a
 * coupling node's interface faces (outward normals of the level's live
 * region) on the level that lies inside the refined box (the other level's
 * coupling nodes keep no face class), 13 otherwise.  Host data only: no
 * device call. */
int acp_node_kind(acp_handle* h, int level, int i, int j, int k, int* id, int* face_class);
/* x-columns of a single-level case's current state in its storage form, for
 * a lattice split into x slabs over several GPUs (one case per slab; the
 * reference runs one lattice on one host, Lattice.cpp:1505-1507, and has no
 * counterpart).  The columns [x0, x0 + ncols) of all 19 populations are
 * packed as [q][k][j][ncols] values of the storage type (8, 4 or 2 bytes):
 * acp_get_columns copies them into buf, acp_put_columns writes them back
 * from buf, and acp_copy_columns copies them from one case straight into
 * another (same ny, nz and storage form; the cases may be on different
 * devices of one process).  buf may be host or device memory.  Each call
 * waits for the cases' queued steps and finishes its copy before returning. */
int acp_get_columns(acp_handle* h, int x0, int ncols, void* buf);
int acp_put_columns(acp_handle* h, int x0, int ncols, const void* buf);
int acp_copy_columns(acp_handle* dst, int dst_x0, acp_handle* src, int src_x0, int ncols);
/* Overwrite a level's populations (both ping-pong arrays) from FP64 f_i. */
int acp_write_populations(acp_handle* h, int level, const double* host_in);
/* Checkpoint / restart of a case's device state.  The reference keeps no
 * restart state: main.cpp:37-121 builds and initialises every run from
 * BoundaryConditions.txt.  A checkpoint file holds the complete state a
 * coarse step reads: both ping-pong population arrays of every level in
 * their storage form (bit-exact), the partner-strain records of the coupling
 * nodes, the ping-pong parity and the number of coarse steps done.
 * acp_checkpoint_save waits for the case's queued steps first.
 * acp_checkpoint_load needs a handle created from a case of the same storage
 * form and level shapes and initialised (acp_init); it then continues bit-for-
 * bit as the saved run would have.  The file names the case it belongs to
 * (storage form with its density shift and FP16 scales, level shapes,
 * operator, equilibrium order, cubic-Mach and MRT options, coupling, layout,
 * restriction and scaling style); a file of another case, or one whose length
 * is not exactly the state's, gives ACP_ERR_INVALID before anything on the
 * device is overwritten.  A read or copy that fails after that point leaves
 * the case's state undefined (ACP_ERR_INVALID / ACP_ERR_CUDA).  Probe series
 * restart empty after a load while the step count continues.  Cases stepped
 * by a batch are refused (ACP_ERR_STATE). */
int acp_checkpoint_save(acp_handle* h, const char* path);
int acp_checkpoint_load(acp_handle* h, const char* path);
/* Legacy structured-points VTK of every level with the fields the reference
 * writes (Lattice::writeResultsVTK, Lattice.cpp:2212-4352: Pressure,
 * Density, Velocity): `<prefix>.vtk` for one level, `<prefix>_level<l>.vtk`
 * for two.  binary = 0 writes ASCII with 8 significant digits (the
 * reference's form); binary = 1 the BINARY form of the same format
 * (big-endian FP64), about a third of the size and read without parsing
 * text.  The four fields of a level are formed on the device in one pass. */
int acp_write_vtk(acp_handle* h, const char* prefix, int binary);
/* A macroscopic field of a level (SI: kg/m^3, m/s, Pa), host buffer of nodes doubles. */
int acp_read_field(acp_handle* h, int level, int field, double* host_out);
/* Pressure probes: n probes at (level, i, j, k) quadruples, i j k in the
 * level's global node indices (fine: twice the coarse ones), on either level;
 * sampled after every coarse step into an FP64 device buffer. */
int acp_set_probes(acp_handle* h, int n, const int* level_ijk);
/* Copy the probe series: out[sample * n + probe] in Pa; *n_samples set to the count. */
int acp_read_probes(acp_handle* h, double* out, int max_samples, int* n_samples);
/* Coarse steps done since acp_init. */
int acp_steps_done(acp_handle* h, long long* steps);
/* Bind the handle to a caller-owned cudaStream_t (NULL: the handle's own). */
int acp_set_stream(acp_handle* h, void* cuda_stream);
/* Device bytes the handle holds. */
int acp_device_bytes(acp_handle* h, size_t* bytes);
/* Device bytes a case would hold, without allocating (admission by HBM footprint). */
int acp_estimate_bytes(const acp_case_desc* d, size_t* bytes);
/* Run n coarse steps kernel by kernel (no graph) with CUDA events between
 * launches and return the average device time per step of each kernel kind:
 * kernel_ms[ACP_K_*].  The per-phase timers the reference lacks (its only
 * timing is wall clock in main.cpp:39-43,126-153). */
enum acp_kernel_kind { ACP_K_MOMENTS = 0, ACP_K_COLLIDE = 1, ACP_K_LODI = 2, ACP_K_COUPLING = 3, ACP_K_PROBES = 4,
                       ACP_K_COUNT = 5 };
int acp_step_timed(acp_handle* h, int n, double* kernel_ms);
/* Kernel launches one coarse step issues (all levels). */
int acp_launches_per_step(acp_handle* h, int* launches);
/* The boundary wiring a case gets (host only, no device needed), one row of
 * 12 integers per boundary node of the coarse level: i j k normalDir n1 n2
 * t1a t1b t2a t2b corner pushMask, neighbours as node indices (k*ny+j)*nx+i
 * or -1, the format the reference's wiring is dumped in for comparison
 * (Lattice::setConnectivity, Lattice.cpp:500-1394).  rows may be NULL to
 * query *count. */
int acp_boundary_wiring(const acp_case_desc* d, long long* rows, long long max_rows, long long* count);
/* Largest window, in nodes, that acp_read_populations_window accepts. */
#define ACP_WINDOW_MAX_NODES 32768
/* Read the populations of the nodes [node_begin, node_begin + node_count) of
 * a level as FP64 f_i into host_out[q * node_count + m] -- the same values
 * acp_read_populations gives for those nodes -- without allocating any device
 * memory.  It has no counterpart in the reference (whose populations live in
 * host memory).  It is for callers that cannot allocate on the device: a
 * serving process that has handed its whole HBM budget to resident lattices,
 * where the temporary FP64 copy of a level that acp_read_populations makes
 * could fail or eat into another solve's share, and applications whose own
 * allocator owns all device memory and forbids cudaMalloc from libraries.
 * The FP64 conversion goes through one fixed device array of
 * ACP_WINDOW_MAX_NODES x 19 doubles (about 5 MB) built into the library; every
 * device that loads the library holds it until the process exits.  Larger
 * windows are rejected (ACP_ERR_INVALID): read a large level window by window.
 * Every call looks up that array's device address in the device's current
 * context (with the handle's device current), so the address stays valid if
 * the application destroys and recreates the context (cudaDeviceReset); the
 * call synchronises the handle's stream, so it is not made inside a stream
 * capture.  All calls share the array: calls that overlap on the GPU (other
 * threads or streams) race and must be serialised by the caller.  Nothing in
 * it needs to start at zero; each call overwrites the part it reads back. */
int acp_read_populations_window(acp_handle* h, int level, long long node_begin, int node_count, double* host_out);
/* ---- batched form --------------------------------------------------------
 * Many initialised cases of uneven sizes, operators, storage forms and
 * refinement layouts advance together: cases with the same kernel templates
 * form a group, each group runs its phases as one persistent launch per phase
 * over all of its cases, groups run side by side, and one coarse step of the
 * whole batch is one CUDA graph launch.  There is no counterpart in the
 * reference, which runs one case per process (main.cpp:37-271).  While a case
 * belongs to a batch, acp_step on it returns ACP_ERR_STATE; the reading calls
 * (acp_sync, acp_read_*) wait for the batch's work.  Results are those of
 * stepping each case alone, to rounding (the same device code, inlined into
 * other kernels, may contract a multiply-add differently). */
typedef struct acp_batch acp_batch;
int acp_batch_create(acp_handle* const* cases, int n, acp_batch** out);
/* n coarse steps of every case, asynchronous on the batch's stream. */
int acp_batch_step(acp_batch* b, int n_coarse_steps);
/* Wait for the batch and report the first case's numeric fault, if any. */
int acp_batch_sync(acp_batch* b);
/* Autotuner: time every candidate schedule (persistent grid of 1/2/4 x the
 * resident blocks or one block per work item; cases in given or descending-
 * size order; tiled z chunk x1 or x2 for 3-D cases) over trial_steps real
 * coarse steps each (the cases advance), keep the fastest and write one line
 * per candidate into report (may be NULL). */
int acp_batch_tune(acp_batch* b, int trial_steps, char* report, size_t report_len);
/* Set the schedule explicitly (persist 0: one block per work item). */
int acp_batch_configure(acp_batch* b, int persist, int largest_first, int chunk_scale);
/* Groups, kernel launches per coarse step, node updates per coarse step. */
int acp_batch_info(acp_batch* b, int* groups, int* launches_per_step, long long* updates_per_step);
/* Releases the batch; its cases stay valid and can be stepped alone again. */
int acp_batch_destroy(acp_batch* b);
const char* acp_batch_last_error(const acp_batch* b);

/* Releases a case (Lattice::~Lattice).  Its device blocks are kept, per
 * device and up to a quarter of the device's memory, for the next case the
 * process creates (an allocation the CUDA driver refuses first gives them back);
 * its page-locked host blocks likewise (up to 1 GiB). */
int acp_destroy(acp_handle* h);
const char* acp_last_error(const acp_handle* h);
const char* acp_status_string(int status);
int acp_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ACP_H */
