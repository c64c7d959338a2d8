/*
 * dnlgpu.h - C ABI of the B200 explicit-dynamics engine for DynELA models.
 *
 * The engine replaces everything below DynELA's `Explicit::solve` for one
 * increment (Sources/dnlFEM/Explicit.C:126-411) and the one-time set-up done by
 * `Model::initSolve` + the pre-loop part of `Explicit::solve`
 * (Sources/dnlFEM/Model.C:360-521, Explicit.C:143-181).  The host side that
 * mirrors DynELA's Python model API (`dnlPython`) fills a `dnl_model_desc`
 * from the script's nodes, elements, material, boundary conditions and solver
 * settings, and drives the engine through the entry points below.
 *
 * Conventions
 *  - plain pointers and sizes only; the caller owns every host array passed in
 *    and may free it as soon as the call returns;
 *  - every entry point returns an int status: 0 (DNL_OK) or a negative
 *    DNL_ERR_* code; the library never calls exit();
 *  - one host thread per handle, one CUDA stream per handle (created by the
 *    engine on the device that is current when dnl_engine_create is called).
 */
#ifndef DNLGPU_H
#define DNLGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Element families on the path (Sources/dnlElements/Element.h type enum). */
enum {
  DNL_ELQUA4NAX = 1, /* 4-node axisymmetric quad, 4 Gauss points (ElQua4NAx.C:21-240) */
  DNL_ELHEX8N3D = 2, /* 8-node hexahedron, 8 Gauss points (ElHex8N3D.C:25-535) */
  DNL_ELQUA4N2D = 3  /* 4-node plane-strain quad, 4 Gauss points (ElQua4N2D.C, Element2D.C:53-99) */
};

/* Critical time step method (Solver.h Courant / PowerIteration). */
enum { DNL_TS_COURANT = 0, DNL_TS_POWER_ITERATION = 1 };

/* Arithmetic of the element pass: FP64 everywhere, or FP32 element math and
 * per-point state with FP64 coordinates, displacements, time and energy sums. */
enum { DNL_PREC_FP64 = 0, DNL_PREC_MIXED = 1 };

/* Constant boundary condition on one node component (BoundaryRestrain.C:98-128,
 * BoundarySpeed.C:139-206); the last condition attached to a component wins. */
enum { DNL_BC_FREE = 0, DNL_BC_RESTRAIN = 1, DNL_BC_SPEED = 2 };

/* Status codes. */
enum {
  DNL_OK = 0,
  DNL_ERR_ARG = -1,            /* invalid argument or size */
  DNL_ERR_CUDA = -2,           /* a CUDA call failed (see dnl_engine_last_error) */
  DNL_ERR_NEG_JACOBIAN = -3,   /* detJ < 0 (ElementPlane.C:75-79, Element3D.C:88-92) */
  DNL_ERR_NEWTON = -4,         /* radial return did not converge (Element.C:560-582) */
  DNL_ERR_POWER_ITERATION = -5,/* power iteration did not converge (Model.C:1002-1005) */
  DNL_ERR_UNSUPPORTED = -6,    /* option not available on this path */
  DNL_ERR_NO_DEVICE = -7       /* no CUDA device / library built without one */
};

/* Per integration point state, component-major: comp*n_ips + ip.
 * Symmetric tensors are stored xx, xy, xz, yy, yz, zz (SymTensor2 _data). */
enum {
  DNL_IP_STRESS = 0,          /* 6 */
  DNL_IP_STRAIN = 6,          /* 6 */
  DNL_IP_PLASTIC_STRAIN = 12, /* 6 */
  DNL_IP_EPSP = 18,           /* equivalent plastic strain */
  DNL_IP_DEPSP = 19,          /* equivalent plastic strain rate */
  DNL_IP_GAMMA = 20,          /* last plastic multiplier */
  DNL_IP_GAMMA_CUM = 21,      /* cumulated plastic multiplier */
  DNL_IP_YIELD = 22,          /* current yield stress */
  DNL_IP_T = 23,              /* temperature */
  DNL_IP_PRESSURE = 24,
  DNL_IP_EINT = 25,           /* specific internal energy */
  DNL_IP_EINEL = 26,          /* specific inelastic energy */
  DNL_IP_DENSITY = 27,
  DNL_IP_DETJ0 = 28,          /* reference detJ (times radius for axisymmetric) */
  DNL_IP_NCOMP = 29
};

/* Nodal fields, each [n_nodes*3] doubles (x, y, z per node). */
enum {
  DNL_NODE_COORDS = 0,
  DNL_NODE_DISP = 1,
  DNL_NODE_U = 2,      /* displacement increment of the last increment (field0->u) */
  DNL_NODE_SPEED = 3,  /* field0->speed */
  DNL_NODE_ACCEL = 4,  /* field0->acceleration */
  DNL_NODE_MASS = 5,   /* lumped mass, repeated on the 3 components */
  DNL_NODE_FORCE = 6,  /* assembled internal force of the last element pass */
  DNL_NODE_SPEED_PREV = 7, /* field1->speed: the speed before the last increment */
  DNL_NODE_U_PREV = 8,     /* field1->u: the displacement increment before the last increment */
  DNL_NODE_ACCEL_PREV = 9  /* field1->acceleration: the acceleration before the last increment */
};
/* The _PREV fields are what the reference's writers read inside an increment:
 * Explicit::endStep (Explicit.C:539-552) writes the history and result files
 * before Model::transfertQuantities swaps field0 and field1, so that their
 * field0 values are those of the start of the increment. */

/* Johnson-Cook elasto-plastic material (Material.h:26-100 + JohnsonCookLaw.C:132-143). */
typedef struct dnl_material {
  double young, poisson, density, heat_capacity, taylor_quinney, T0;
  double A, B, C, n, m, depsp0, Tm, Tref; /* Johnson-Cook A, B, C, n, m, eps0_dot, Tm, T0 */
} dnl_material;

/* Piecewise-linear time function (DiscreteFunction.C:188-213); x strictly increasing. */
typedef struct dnl_function {
  int32_t n_points;
  const double *x;
  const double *y;
} dnl_function;

/* One model (one simulation instance). */
typedef struct dnl_model_desc {
  int32_t elem_type;           /* DNL_ELQUA4NAX, DNL_ELHEX8N3D or DNL_ELQUA4N2D */
  int32_t n_nodes;
  int32_t n_elems;
  const double *coords;        /* [n_nodes*3] */
  const int32_t *conn;         /* [n_elems*nodes_per_element], 0-based node indices */
  const int32_t *elem_mat;     /* [n_elems] material index, or NULL (all 0) */
  int32_t n_materials;
  const dnl_material *materials;
  const double *v_init;        /* [n_nodes*3] initial speed (BoundarySpeed::applyInitial), or NULL */
  const int8_t *bc_code;       /* [n_nodes*3] DNL_BC_*, or NULL (all free) */
  const double *bc_value;      /* [n_nodes*3] imposed speed for DNL_BC_SPEED, or NULL */
  const int32_t *bc_func;      /* [n_nodes*3] function index scaling bc_value, -1 none, or NULL */
  int32_t n_functions;
  const dnl_function *functions;
  double t_start, t_end;       /* Solver::setTimes */
  int32_t ts_method;           /* DNL_TS_* */
  int32_t ts_freq;             /* Solver::setComputeTimeStepFrequency (default 10) */
  double ts_safety;            /* Solver::setTimeStepSafetyFactor (default 0.9) */
  double rho_b;                /* Explicit::setDissipation (default 0.8182) */
  int32_t precision;           /* DNL_PREC_* */
  int32_t stress_method;       /* DNL_STRESS_*: DynELA::setStressComputation (DynELA.C:1407-1431) */
  int32_t node_order;          /* DNL_ORDER_*: how the engine numbers its copy of the nodes */
} dnl_model_desc;

/* Node numbering inside the engine.  The element pass gathers each element's
 * nodes, so nodes that share elements should be close in memory.  GIVEN keeps
 * the caller's numbering; RCM renumbers by reverse Cuthill-McKee
 * (dnl_mesh_order_rcm); AUTO takes RCM when it at least halves the mean
 * element span (dnl_mesh_span) of the given numbering.  Whatever the choice,
 * every node index and node array of this interface stays in the caller's
 * numbering; the results are the same bits up to the order of the sums over
 * nodes (energies, the power-iteration time step's norms). */
enum { DNL_ORDER_GIVEN = 0, DNL_ORDER_RCM = 1, DNL_ORDER_AUTO = 2 };

/* Reverse Cuthill-McKee ordering of a mesh's nodes (host code, no device
 * needed): order[k] is the node numbered k.  conn: [n_elems*npe], npe 4 or 8. */
int dnl_mesh_order_rcm(int32_t n_nodes, int32_t n_elems, int32_t npe, const int32_t *conn, int32_t *order);
/* Mean over the elements of (largest - smallest node number) under the
 * numbering order[k] = node numbered k (NULL: the given numbering). */
int dnl_mesh_span(int32_t n_nodes, int32_t n_elems, int32_t npe, const int32_t *conn, const int32_t *order,
                  double *mean_span);

/* Radial return of Model::computeStress (Model.C:840-851): the
 * Newton-Raphson iteration of Element::computeStress (Element.C:407-622) or
 * the one-step return of Element::computeStressDirect (Element.C:625-850). */
enum { DNL_STRESS_NEWTON = 0, DNL_STRESS_DIRECT = 1 };

/* Solver state of one instance. */
typedef struct dnl_control {
  double time;        /* Model::currentTime */
  double time_step;   /* Solver::timeStep (after the clip to the end time) */
  double t_end;
  int64_t increment;  /* Solver::currentIncrement */
  int32_t status;     /* DNL_OK or DNL_ERR_* raised on the device */
  int32_t bad_index;  /* element (negative detJ) or integration point (Newton) that failed */
  int32_t done;       /* time >= t_end */
  int32_t fp64_resolves; /* mixed path: points re-solved in FP64 during the last run call */
  double last_time_step; /* time step of the last completed increment (Solver::timeStep as the
                            history files see it in Explicit::endStep, Explicit.C:539-552) */
} dnl_control;

typedef struct dnl_engine dnl_engine;

/* Returns the number of CUDA devices visible (0 when none), never fails. */
int dnl_device_count(void);

/* Create an engine for one model.  Uploads the description to the current
 * device.  Replaces DynELA::initSolve -> Model::initSolve (Model.C:360-521)
 * data layout set-up. */
int dnl_engine_create(const dnl_model_desc *desc, dnl_engine **out);

/* Create one engine that advances n independent models together (batched
 * mode): one element pass, one nodal pass and one time-step pass per step for
 * all of them, each with its own time, time step and material. */
int dnl_engine_batch_create(const dnl_model_desc *const *descs, int32_t n, dnl_engine **out);

int dnl_engine_destroy(dnl_engine *h);

/* Text of the last error raised on this handle (or the last create error when h is NULL). */
const char *dnl_engine_last_error(const dnl_engine *h);

/* One-time start of the solve: reference Jacobian, lumped mass, first time
 * step, first element pass (Explicit.C:143-181 + Model::computeMassMatrix,
 * Model.C:537-592). */
int dnl_engine_init(dnl_engine *h);

/* Advance every unfinished instance until its time reaches min(t_pause, t_end)
 * or max_incs increments have been run in this call (max_incs <= 0: no limit).
 * Replaces the increment loop of Explicit::solve (Explicit.C:184-256).
 * *incs_done (may be NULL) receives the largest number of increments run by
 * one instance in this call.  An instance whose increment fails (negative
 * Jacobian, radial return without convergence) stops there with the error in
 * its dnl_control.status, where the reference would abort the whole solve;
 * the other instances of a batch go on, and once every instance has stopped
 * the call returns the error of the lowest-numbered failed instance. */
int dnl_engine_run(dnl_engine *h, double t_pause, int64_t max_incs, int64_t *incs_done);

/* Kernel-level entry point: one element pass (strains, pressure, radial
 * return, final rotation, internal forces and their assembly; Explicit.C:204-226)
 * on the current state with the given time step, without the nodal update.
 * Instance 0 only. */
int dnl_engine_element_pass(dnl_engine *h, double time_step);

/* Number of instances, nodes, elements and integration points (all instances). */
int dnl_engine_sizes(const dnl_engine *h, int32_t *n_instances, int32_t *n_nodes,
                     int32_t *n_elems, int32_t *n_ips);

/* First node / element / integration point of instance i in the concatenated arrays. */
int dnl_engine_instance_offsets(const dnl_engine *h, int32_t i, int32_t *node0,
                                int32_t *elem0, int32_t *ip0);
/* The numbering the engine chose for instance i's nodes: DNL_ORDER_GIVEN or
 * DNL_ORDER_RCM. */
int dnl_engine_node_order(const dnl_engine *h, int32_t instance, int32_t *order);

int dnl_engine_control(const dnl_engine *h, int32_t instance, dnl_control *out);

/* Copy one nodal field (DNL_NODE_*) of all instances to host memory [n_nodes*3]. */
int dnl_engine_get_nodes(dnl_engine *h, int32_t field, double *out);
/* Overwrite one nodal field (coords, disp, u, speed, accel) from host memory. */
int dnl_engine_set_nodes(dnl_engine *h, int32_t field, const double *in);

/* Copy / overwrite the integration-point state, [DNL_IP_NCOMP * n_ips] doubles
 * component-major (converted from/to FP32 on the mixed path). */
int dnl_engine_get_ips(dnl_engine *h, double *out);
int dnl_engine_set_ips(dnl_engine *h, const double *in);
/* The point state in the precision the engine keeps it in, same layout:
 * word = 4 (float) on the mixed path, 8 (double) on the FP64 path; another
 * word size returns DNL_ERR_ARG.  Nothing is widened, so the mixed path's
 * state crosses to the host in half the bytes of dnl_engine_get_ips. */
int dnl_engine_get_ips_native(dnl_engine *h, void *out, int32_t word);

/* History items (replaces the per-save reads of HistoryFile::save,
 * HistoryFile.C:289-317, and of the Field extraction it calls,
 * Element.C:1195-1240, Model.C:612-626): the values a history file needs at a
 * save time are selected on the device and only they cross to the host.
 * An item is one of
 *   DNL_ITEM_NODE     3 doubles: nodal field `field` (DNL_NODE_*) of node `index`
 *   DNL_ITEM_POINT    DNL_IP_NCOMP doubles: the state of integration point `index`
 *   DNL_ITEM_KINETIC  1 double: kinetic energy of instance `index` on speed
 *                     field `field` (DNL_NODE_SPEED or DNL_NODE_SPEED_PREV),
 *                     fixed-order FP64 sum of m |v|^2 / 2.
 * dnl_engine_set_items checks and uploads the list (replacing a previous one)
 * and returns the number of doubles one gather writes; dnl_engine_gather_items
 * writes them, item after item in list order, to `out`. */
enum
{
  DNL_ITEM_NODE = 0,
  DNL_ITEM_POINT = 1,
  DNL_ITEM_KINETIC = 2
};
typedef struct
{
  int32_t kind, field, index, reserved;
} dnl_item;
int dnl_engine_set_items(dnl_engine *h, const dnl_item *items, int32_t n, int64_t *n_values);
int dnl_engine_gather_items(dnl_engine *h, double *out);

/* History records kept on the device, so that a run does not stop at save
 * times (single models).  Each schedule follows HistoryFile::save
 * (HistoryFile.C:292-317): at the end of every increment, after the time
 * update (Explicit::endStep, Explicit.C:539-552), it is due when
 * !(time > start && time < next), and next then moves on by save.  An
 * increment with a schedule due appends one record to a ring of `capacity`
 * records on the device (0: 64): DNL_HIST_HEAD doubles — time, increment,
 * the increment's time step, the mask of the due schedules as two 32-bit
 * halves (schedule j is bit j, j < 64) — then the values of the items of
 * dnl_engine_set_items, as dnl_engine_gather_items lays them out.  Runs
 * look at the device at least every `capacity` increments and move the
 * records to the host; dnl_engine_history_records hands them out, oldest
 * first (out = NULL: only the number waiting).  Calling dnl_engine_set_items
 * again stops the records (their width changes); n = 0 stops them.  No
 * counterpart in the reference, which writes its history files on the host
 * inside every increment. */
#define DNL_HIST_HEAD 5
typedef struct dnl_history_schedule {
  double start, next, save; /* HistoryFile _startTime, _nextTime, _saveTime */
} dnl_history_schedule;
int dnl_engine_set_history(dnl_engine *h, const dnl_history_schedule *schedules, int32_t n, int32_t capacity);
int dnl_engine_history_records(dnl_engine *h, double *out, int64_t max_records, int64_t *n_records);

/* Nodal values of point-state quantities, extracted as the reference does for
 * its node fields and result files (Node::fieldScalar / fieldSymTensor2,
 * Node.C:244-365): at each node, the values of the Gauss points of every
 * element around it, extrapolated to the node (ElementData
 * integrationPointsToNode, ElHex8N3D.C:40-90, ElQua4NAx.C:37-58), summed
 * and divided by the number of those elements, in FP64.  comps[k] is a
 * point-state component DNL_IP_* or DNL_NODE_AVG_VON_MISES (the von Mises
 * stress of each point, SymTensor2::vonMises).  out: [n][n_nodes] doubles,
 * all instances. */
#define DNL_NODE_AVG_VON_MISES 64
int dnl_engine_node_averages(dnl_engine *h, const int32_t *comps, int32_t n, double *out);

/* Result file of one instance in the reference's format (DynELA::writeVTKFile
 * -> VtkInterface::write, DynELA.C:688-711, VtkInterface.C:68-221): legacy
 * ASCII VTK unstructured grid with the title, the time, the nodes, the cells
 * and, as point data, the fields listed (DNL_VTK_*, in the list's order),
 * numbers printed as the reference's streams print them (6 significant
 * digits).  prev = 1 writes the displacement increments, speeds and
 * accelerations of before the last increment, which is what the reference's
 * files written inside an increment hold (Explicit::endStep writes them
 * before the field swap); prev = 0 the current ones (its initial and final
 * files).  No counterpart for the field list's storage: the reference reads
 * it from its settings file (VtkFields, VtkInterface::initFields). */
enum {
  /* nodal vectors (Node::fieldVec3D, Node.C:380-401) */
  DNL_VTK_COORDS = 0, DNL_VTK_DISP = 1, DNL_VTK_DISP_INC = 2, DNL_VTK_SPEED = 3, DNL_VTK_SPEED_INC = 4,
  /* point-state scalars averaged at the nodes (Node::fieldScalar) */
  DNL_VTK_DENSITY = 5, DNL_VTK_GAMMA = 6, DNL_VTK_GAMMA_CUMULATE = 7, DNL_VTK_INTERNAL_ENERGY = 8,
  DNL_VTK_PLASTIC_STRAIN = 9, DNL_VTK_PLASTIC_STRAIN_RATE = 10, DNL_VTK_PRESSURE = 11, DNL_VTK_T = 12,
  DNL_VTK_VON_MISES = 13, DNL_VTK_YIELD = 14, DNL_VTK_MASS = 15,
  /* point-state tensors averaged at the nodes (Node::fieldSymTensor2) */
  DNL_VTK_PLASTIC_STRAIN_TENSOR = 16, DNL_VTK_STRAIN_TENSOR = 17, DNL_VTK_STRESS_TENSOR = 18,
  DNL_VTK_NFIELDS = 19
};
int dnl_engine_write_vtk(dnl_engine *h, int32_t instance, const char *path, const char *title,
                         const int32_t *fields, int32_t n_fields, int32_t prev);

/* Energies of one instance, FP64 sums: [0] kinetic (Model.C:612-626, field0
 * speeds), [1] internal = sum rho0*detJ0*w*e_int (x 2 pi for axisymmetric),
 * [2] inelastic (plastic work), same weights. */
int dnl_engine_energies(dnl_engine *h, int32_t instance, double out[3]);

/* Device-side time of the kernels of the last dnl_engine_run call, in ms:
 * [0] element pass, [1] nodal pass, [2] time-step pass, [3] whole run. Only
 * filled when timing was enabled with dnl_engine_set_timing(h, 1): the
 * increments then run kernel by kernel (no graph), queued in chunks of up to
 * 64 with CUDA events around each pass that are read after the chunk, so
 * that no bracket holds host launch latency; the run stops at the end of
 * the chunk in which its instances stop (the increments past the stop do
 * nothing and add a few microseconds each to the sums). */
int dnl_engine_set_timing(dnl_engine *h, int32_t on);
int dnl_engine_timings(const dnl_engine *h, double out[4]);

/* Increments captured in one CUDA graph replay (1..64, default 8): with
 * more, the first kernel of an increment is scheduled while the previous
 * increment's last kernel ends (programmatic serialization inside the graph)
 * instead of after a replay boundary (1.2 % per increment on the
 * 153,600-element bar from 1 to 8).  A run stops on the same increment
 * either way: the increments past an instance's stop do nothing. */
int dnl_engine_set_graph_increments(dnl_engine *h, int32_t n);

/* Number of kernel launches issued on the device by the last run call. */
int64_t dnl_engine_launch_count(const dnl_engine *h);

/* Element-pass autotuner (hex8 models): times each kernel variant (staging
 * scheme: plain, bulk-copied point state, or every input staged; register
 * budget; points per block for the plain kernel: 64, 128 or 256, i.e. 8, 16
 * or 32 hexahedra; names from dnl_variant_name) over `steps` increments
 * run from a saved copy of the state, keeps the fastest for the following runs
 * (on the mixed path a preferred variant when it is within 1 % of the fastest,
 * as it holds up best later in an impact: the plain pass on 64-point blocks,
 * 9, for a single model, the staged 4-blocks-per-SM pass, 5, for a batch) and
 * restores the state.  A batch (several instances) is offered the
 * persistent variants only (its ms entries for the plain ones are -1): the
 * plain variants launch a block per tile of the whole batch at every
 * increment, even when few instances still run.  No counterpart in the
 * reference (its element loop has one implementation). */
int dnl_engine_autotune(dnl_engine *h, int32_t steps);
#define DNL_NUM_VARIANTS 12
/* Variant in use and the element-pass time (ms) the autotuner measured for each. */
int dnl_engine_variant(const dnl_engine *h, int32_t *variant, double ms[DNL_NUM_VARIANTS]);
/* Force an element-pass variant (0 .. DNL_NUM_VARIANTS-1). */
int dnl_engine_set_variant(dnl_engine *h, int32_t variant);
/* Name of a variant of the precision's list ("stage/4": staged tiles, a
 * register budget of 4 blocks of 128 threads per SM), or NULL. */
const char *dnl_variant_name(int32_t precision, int32_t variant);

/* Element pass that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc (a host application
 * whose own memory manager owns the GPU, or code between stream captures where
 * an allocation would synchronize the device): every input and output is a
 * caller-owned device array, and the scratch (per element-node force slots,
 * node -> slot lists, a control block) is a static device array of about
 * 5.3 MB that every GPU loading the library keeps until the process exits.
 * One call = strains, pressure, radial return, final rotation, density and the
 * nodal internal forces (the same element pass as dnl_engine_element_pass) in
 * FP64 for a model of at most DNL_STATIC_MAX_ELEMS elements and
 * DNL_STATIC_MAX_NODES nodes; larger sizes return DNL_ERR_ARG.
 *   d_coords, d_du [n_nodes*3]: current coordinates and displacement increment
 *   d_conn [n_elems*nodes_per_element]: 0-based connectivity
 *   d_ips [DNL_IP_NCOMP*n_ips] FP64 component-major point state, updated in place
 *   d_force [n_nodes*3]: assembled internal forces (output)
 *   stream: a cudaStream_t (NULL: the default stream); the call waits for it at the end.
 * The first call on a device looks up the scratch address: make it before any
 * stream capture.  All calls share the scratch, so calls that overlap on the
 * GPU (other streams, other threads) race: serialise them. */
#define DNL_STATIC_MAX_ELEMS 16384
#define DNL_STATIC_MAX_NODES 65536
int dnl_element_pass_static(int32_t elem_type, int32_t n_nodes, int32_t n_elems, const double *d_coords,
                            const double *d_du, const int32_t *d_conn, const dnl_material *material,
                            double time_step, double *d_ips, double *d_force, void *stream);

/* ------------------------------------------------------------------------
 * Learned Newton initial guess of the radial return.  No counterpart in the
 * reference (its return starts from the previous increment's gamma,
 * Element.C:507-515).  A 5 -> 64 -> 64 -> 64 -> 1 SiLU network maps the trial
 * state of a yielding Gauss point to r = gamma / gamma_max, with gamma_max =
 * (sigma_trial - sigma_y) / (sqrt(3/2) 2G) the upper end of the bracket the
 * return starts with (a yield stress that falls during the increment can take
 * gamma past it).  The return starts from min(max(r, 0), 2) * gamma_max and
 * keeps its own bracket and stopping tests, so it converges to the same root
 * (the network only changes the iterations).
 * Inputs, computed in FP32 from the point state before the return:
 *   x0 = sigma_trial / A, x1 = eps_p, x2 = ln(1 + depsp / depsp0),
 *   x3 = T / Tm, x4 = ln(3 G dt depsp0 / A)
 * and normalised as (x - in_mean) * in_scale, then, when in_clip > 0, held to
 * [-in_clip, in_clip] (inputs past the range the network was trained on are
 * taken at its edge instead of extrapolated).  The hidden layers run as BF16
 * tensor-core products with FP32 accumulation; the output layer in FP32.
 * Weights are FP32 here and rounded to BF16 on the device. */
#define DNL_MLP_IN 5
#define DNL_MLP_HIDDEN 64
typedef struct dnl_mlp {
  float w1[DNL_MLP_HIDDEN][16]; /* inputs 5..15 unused (zero) */
  float b1[DNL_MLP_HIDDEN];
  float w2[DNL_MLP_HIDDEN][DNL_MLP_HIDDEN];
  float b2[DNL_MLP_HIDDEN];
  float w3[DNL_MLP_HIDDEN][DNL_MLP_HIDDEN];
  float b3[DNL_MLP_HIDDEN];
  float w4[DNL_MLP_HIDDEN];
  float b4;
  float in_mean[DNL_MLP_IN];
  float in_scale[DNL_MLP_IN];
  float out_exp; /* 0: r = output; 1: r = exp(output) (a network trained on ln r) */
  float in_clip; /* > 0: normalised inputs held to [-in_clip, in_clip]; 0: not held */
} dnl_mlp;

/* One training pair as harvested from the radial return: the 5 raw inputs,
 * the target r, the converged gamma and gamma_max. */
#define DNL_MLP_PAIR_WORDS 8

/* Element-pass mode of the engine (mixed precision, hex8 and axisymmetric):
 * DNL_MODE_PLAIN the tuned variants; DNL_MODE_STATS the same return with its
 * Newton iterations counted; DNL_MODE_HARVEST counting + training pairs
 * written to the buffer of dnl_engine_set_harvest; DNL_MODE_GUESS counting +
 * the network of dnl_engine_set_guess_network as the first iterate. */
enum { DNL_MODE_PLAIN = 0, DNL_MODE_STATS = 1, DNL_MODE_HARVEST = 2, DNL_MODE_GUESS = 3 };
int dnl_engine_set_mode(dnl_engine *h, int32_t mode);
int dnl_engine_set_guess_network(dnl_engine *h, const dnl_mlp *net);
/* d_pairs: caller-owned device array of capacity*DNL_MLP_PAIR_WORDS floats; one
 * yielding point of the guess scope (dnl_engine_set_guess_scope) in `stride`
 * (chosen by a hash of point and increment) is kept until the buffer is full.
 * Resets the pair count. */
int dnl_engine_set_harvest(dnl_engine *h, float *d_pairs, int64_t capacity, int32_t stride);
/* Points that passed the stride since the last dnl_engine_set_harvest: the
 * pairs stored are the first min(count, capacity) rows of the buffer. */
int dnl_engine_harvest_count(dnl_engine *h, int64_t *count);
/* Which yielding points start from the network in DNL_MODE_GUESS:
 * DNL_GUESS_ALL every one, DNL_GUESS_FIRST_YIELD only those without a
 * previous gamma to start from (eps_p = 0, where the reference starts from
 * gamma = 1e-8); the others keep the warm start. */
enum { DNL_GUESS_ALL = 0, DNL_GUESS_FIRST_YIELD = 1 };
int dnl_engine_set_guess_scope(dnl_engine *h, int32_t scope);
/* Since the last reset (counting modes): [0] yield-function evaluations of
 * the returns and [1] yielding points; [2] yielding points of the guess scope
 * and [3] their evaluations (in DNL_MODE_GUESS, the points that started from
 * the network). */
int dnl_engine_newton_stats(dnl_engine *h, int64_t out[4], int32_t reset);

/* Network kernels (BF16 tensor-core products, FP32 accumulation), on
 * caller-owned device arrays, on `stream` (NULL: default), synchronous.
 * d_x [n*5] raw inputs, d_y [n] outputs. */
int dnl_mlp_forward(const dnl_mlp *net, const float *d_x, int64_t n, float *d_y, void *stream);
/* Gradient of the mean squared error (1/n) sum (y - t)^2 over n samples
 * (d_t [n]) with respect to every weight and bias, into *grad (host); *loss
 * receives the mean squared error.  in_mean / in_scale are not trained. */
int dnl_mlp_gradients(const dnl_mlp *net, const float *d_x, const float *d_t, int64_t n, dnl_mlp *grad,
                      float *loss, void *stream);
/* Adam training (FP32 master weights, BF16 products) on n pairs d_x / d_t:
 * `epochs` passes over a seeded shuffle in minibatches of batch_tiles*128
 * pairs.  *net is the initial network on entry and the trained one on return;
 * loss_history [epochs] (host, may be NULL) receives each epoch's mean loss. */
int dnl_mlp_train(dnl_mlp *net, const float *d_x, const float *d_t, int64_t n, int32_t epochs, int32_t batch_tiles,
                  float learning_rate, uint64_t seed, float *loss_history, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DNLGPU_H */
