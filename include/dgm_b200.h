/*
 * dgm_b200.h -- C ABI of the B200 (sm_100a) DG residual + SSP-RK3 library.
 *
 * Drop-in boundary for DGM_in_rust's hot path.  A host (the Rust FFI crate, Python ctypes,
 * C++) passes the already-processed mesh, basis/quadrature tables and parameters once, then
 * calls the entry points below in place of the reference's methods.  Arrays crossing the
 * boundary use the reference's own layout: states and residuals are Array<f64, Ix3>
 * [element][variable][basis] in C order (initialization.rs:70-71).  No torch types, no
 * ownership transfer: the caller keeps every pointer it passes.
 *
 * Error convention: every entry point returns a DGM_* status.  The reference panics in these
 * cases (flux.rs:56-61 via spatial_disc.rs:195-200; weno.rs:107); the FFI crate maps a non-OK
 * status to panic!(dgm_status_string(status)).  dgm_error_location() gives the edge or element
 * the device flagged first.
 *
 * Threading: a context is not thread-safe; it owns one CUDA stream and device-resident
 * buffers.  One context per mesh instance.  There is no CPU fallback: without a usable
 * CUDA device dgm_create fails with DGM_NO_DEVICE.
 */
#ifndef DGM_B200_H
#define DGM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------- */
#define DGM_OK 0
#define DGM_NEG_DENSITY 1             /* "Negative density found in HLLC!"  flux.rs:56-57   */
#define DGM_NEG_PRESSURE 2            /* "Negative pressure found in HLLC!" flux.rs:59-60   */
#define DGM_NONFINITE 3               /* non-finite time step                                */
#define DGM_TOO_MANY_BOUNDARY_EDGES 4 /* "Invalid number of boundary neighbours!" weno.rs:107 */
#define DGM_OOM 5                     /* device allocation failed                           */
#define DGM_TIMEOUT 6                 /* a bounded device wait gave up                      */
#define DGM_BAD_ARG 7                 /* unsupported order/rule, bad sizes or pointers       */
#define DGM_CUDA_ERROR 9              /* a CUDA runtime call failed                         */
#define DGM_NO_DEVICE 10              /* no usable CUDA device                              */
#define DGM_NOT_READY 11              /* dgm_query: work still in flight (not an error)     */
#define DGM_LIST_OVERFLOW 12          /* a limiter worklist reached its capacity: the entry   */
                                      /* was dropped, the pass's results are not valid        */

/* ---- boundary types (mesh.rs:174-178) ---------------------------------------------------- */
#define DGM_WALL 0
#define DGM_FARFIELD 1

/* Processed mesh, i.e. the fields of Mesh/Element/Edge/Patch (mesh.rs:5-189) as they stand
 * after process_mesh and the Mesh::compute_* calls (initialization.rs:40-66).  All arrays are
 * dense, 0-based, C order. */
typedef struct dgm_mesh_desc {
  int64_t n_vertices;
  int64_t n_elements;
  int64_t n_edges;
  int64_t n_patches;
  const double* vertex_xy;          /* [n_vertices][2]            Vertex {x, y}             */
  const int64_t* elem_vertices;     /* [n_elements][3]            Element::ivertices        */
  const int64_t* elem_edges;        /* [n_elements][3]            Element::iedges           */
  const int64_t* elem_neighbours;   /* [n_elements][3], -1 = none Element::ineighbours      */
  const double* elem_jacob_det;     /* [n_elements]               Element::jacob_det        */
  const double* elem_circumradius;  /* [n_elements]               Element::circumradius     */
  const double* elem_minimum_height;/* [n_elements]               Element::minimum_height   */
  const int64_t* edge_elements;     /* [n_edges][2], [1] = -1 on the boundary  Edge::ielements */
  const int64_t* edge_vertices;     /* [n_edges][2]               Edge::ivertices           */
  const int64_t* edge_in_cell;      /* [n_edges][2]               Edge::in_cell_indices     */
  const double* edge_jacob_det;     /* [n_edges]                  Edge::jacob_det (length)  */
  const double* edge_normal;        /* [n_edges][2]               Edge::normal              */
  const int64_t* edge_patch;        /* [n_edges], -1 = internal   Edge::ipatch              */
  const int32_t* patch_type;        /* [n_patches] DGM_WALL / DGM_FARFIELD  Patch::boundary_type */
  const double* patch_quantity;     /* [n_patches][4] rho,u,v,p (far field)  BoundaryQuantity */
  int64_t n_internal_edges;
  const int64_t* internal_edges;    /* Mesh::internal_edge_indices                          */
  int64_t n_boundary_elements;
  const int64_t* boundary_elements; /* Mesh::boundary_element_indices                       */
} dgm_mesh_desc;

/* Host mesh preprocessing, native (no device memory, no GPU needed): process_mesh
 * (initialization.rs:112-261) and the Mesh::compute_* geometry (mesh.rs:15-147) in one pass that
 * is linear in the mesh size, producing the arrays of dgm_mesh_desc bit for bit as the reference
 * computes them.  Input: what GmshParser::parse (mesh_parser.rs:28-158) returns -- vertices, the
 * node pairs of every boundary line block concatenated in block order, and the triangles of every
 * surface block concatenated in block order, all 0-based.  dgm_mesh_process returns a handle
 * (NULL with *status set on failure: DGM_BAD_ARG for a node index out of range); dgm_mesh_counts
 * gives the array sizes (edges, internal edges, internal elements; the boundary elements are the
 * rest); dgm_mesh_fetch copies the arrays into caller-allocated buffers (any pointer may be NULL);
 * dgm_mesh_free releases the handle.  Patch types and quantities stay with the caller (one per
 * boundary block). */
typedef struct dgm_mesh_build dgm_mesh_build;
dgm_mesh_build* dgm_mesh_process(int64_t n_vertices, const double* vertex_xy, int64_t n_boundary_edges,
                                 const int64_t* boundary_pairs /* [n_boundary_edges][2] */, int64_t n_elements,
                                 const int64_t* elem_vertices /* [n_elements][3] */, int32_t* status);
int32_t dgm_mesh_counts(const dgm_mesh_build* m, int64_t* n_edges, int64_t* n_internal_edges,
                        int64_t* n_internal_elements);
int32_t dgm_mesh_fetch(const dgm_mesh_build* m, int64_t* elem_edges /* [ne][3] */,
                       int64_t* elem_neighbours /* [ne][3] */, double* elem_jacob_det /* [ne] */,
                       double* elem_circumradius /* [ne] */, double* elem_minimum_height /* [ne] */,
                       int64_t* edge_elements /* [n_edges][2] */, int64_t* edge_vertices /* [n_edges][2] */,
                       int64_t* edge_in_cell /* [n_edges][2] */, double* edge_jacob_det /* [n_edges] */,
                       double* edge_normal /* [n_edges][2] */, int64_t* internal_edges,
                       int64_t* internal_elements, int64_t* boundary_elements);
void dgm_mesh_free(dgm_mesh_build* m);

/* gmsh 4.1 ASCII reader with the reference's line state machine (GmshParser::parse,
 * mesh_parser.rs:28-158), native.  dgm_gmsh_parse reads the file (NULL with *status set on
 * failure: DGM_BAD_ARG where the reference's parse panics -- a missing file, a malformed number,
 * an entity without a physical name); dgm_gmsh_counts gives the number of vertices, boundary line
 * blocks (dim 1) and triangle blocks (dim 2); dgm_gmsh_vertices copies [n_vertices][2];
 * dgm_gmsh_block_size gives the pairs (dim 1) or triangles (dim 2) of block i, -1 if none;
 * dgm_gmsh_block copies its 0-based node ids; dgm_gmsh_block_name gives a line block's physical
 * name (valid until dgm_gmsh_free). */
typedef struct dgm_gmsh dgm_gmsh;
dgm_gmsh* dgm_gmsh_parse(const char* path, int32_t* status);
int32_t dgm_gmsh_counts(const dgm_gmsh* g, int64_t* n_vertices, int32_t* n_edge_blocks, int32_t* n_elem_blocks);
int32_t dgm_gmsh_vertices(const dgm_gmsh* g, double* vertex_xy);
int64_t dgm_gmsh_block_size(const dgm_gmsh* g, int32_t dim, int32_t i);
const char* dgm_gmsh_block_name(const dgm_gmsh* g, int32_t i);
int32_t dgm_gmsh_block(const dgm_gmsh* g, int32_t dim, int32_t i, int64_t* node_ids);
void dgm_gmsh_free(dgm_gmsh* g);

/* write_to_vtk (write_results.rs:8-93), native, on the host: the legacy ASCII VTK file the
 * reference writes through vtkio (points with z = 0, triangles, cell data Density, Velocity
 * (u, v, 0), Pressure), numbers as Rust prints an f64 with {}.  fields is [n_elements][4] =
 * density, x velocity, y velocity, pressure (dgm_cell_fields gives them from the device state).
 * The directory must exist.  DGM_BAD_ARG when the file cannot be written. */
int32_t dgm_vtk_write(const char* path, int64_t n_vertices, const double* vertex_xy /* [n_vertices][2] */,
                      int64_t n_elements, const int64_t* elem_vertices /* [n_elements][3] */,
                      const double* fields /* [n_elements][4] */);

/* Basis and quadrature tables: DubinerBasis (basis_function.rs:6-13) and GaussPoints
 * (gauss_point.rs:4-11).  Supported (order, cell rule, edge rule): (1,3,2), (2,6,3), (3,12,4). */
typedef struct dgm_tables_desc {
  int32_t order;                    /* SolverParameters::order_of_polynomials               */
  int32_t n_basis;                  /* number_of_basis_functions                            */
  int32_t n_cell_gp;                /* number_of_cell_gp                                    */
  int32_t n_edge_gp;                /* number_of_edge_gp                                    */
  int32_t n_deriv_keys;             /* keys in dphi_cell_ref: (order+1)(order+2)/2 - 1, >= 2 */
  int32_t _pad;
  const double* cell_weights;       /* [n_cell_gp]                                          */
  const double* edge_weights;       /* [n_edge_gp]                                          */
  const double* phi_cell;           /* [n_cell_gp][n_basis]       phis_cell_gps             */
  const double* phi_edge;           /* [3][n_edge_gp][n_basis]    phis_edge_gps             */
  /* Reference-space derivatives d^a/dxi^a d^b/deta^b of each mode at the cell points,
   * [n_cell_gp][n_basis][n_deriv_keys], keys ordered (1,0),(0,1),(2,0),(1,1),(0,2),(3,0),...
   * (the HashMap keys of dphis_cell_gps, basis_function.rs:114-151). */
  const double* dphi_cell_ref;
  const double* mass_diag;          /* [n_basis]                  mass_mat_diag             */
} dgm_tables_desc;

typedef struct dgm_params {
  double hcr;                       /* FlowParameters::hcr (ratio of specific heats)        */
  double cfl;                       /* SolverParameters::cfl                                */
  double final_time;                /* SolverParameters::final_time                         */
  int64_t final_step;               /* SolverParameters::final_step                         */
  int32_t limiter;                  /* 1 = WENO/KXRCF limiter after each stage (reference), 0 = off */
  int32_t device;                   /* CUDA device ordinal                                  */
  /* 0 = FP64 throughout (the reference's arithmetic); 1 = FP32 state, contractions, fluxes and
   * stage updates, with the limiter, the HLLC positivity checks, the time step and the
   * diagnostics kept in FP64; 2 = as 1 with the element pass's two basis contractions
   * (basis -> quadrature points, quadrature and edge points -> basis) on the tensor cores
   * (tcgen05, TF32 operands, FP32 accumulation); 3 = as 2 with each operand split into a TF32
   * head and tail (three products: FP32-level accuracy); 4 = FP64 state with FP32 contractions,
   * fluxes and residuals (FP32 edge fluxes), the stage combinations, limiter, positivity checks,
   * time step and diagnostics in FP64: the state does not round to FP32 each stage.  No
   * counterpart in the reference. */
  int32_t precision;
  int32_t _reserved;
} dgm_params;

typedef struct dgm_ctx dgm_ctx;

/* Build a device-resident solver context (the GPU side of Solver/SpatialDisc/TemperalDisc,
 * solver.rs:32-43, spatial_disc.rs:17-25, temporal_disc.rs:8-19).  Copies everything it needs;
 * the descriptors may be freed after the call.  *status receives DGM_OK or an error. */
dgm_ctx* dgm_create(const dgm_mesh_desc* mesh, const dgm_tables_desc* tables,
                    const dgm_params* params, int32_t* status);
void dgm_destroy(dgm_ctx* ctx);

/* SpatialDisc::compute_residuals(&self, residuals: &mut Array3, solutions: &Array3)
 * (src/spatial_disc.rs:27).  Same semantics: residuals = (residuals + volume + edge +
 * boundary terms) / mass, host buffers of n_elements*4*n_basis doubles. */
int32_t dgm_compute_residuals(dgm_ctx* ctx, double* residuals, const double* solutions);

/* SpatialDisc::apply_limiter(&self, solutions: &mut Array3) (src/spatial_disc/limiter.rs:7):
 * modified-KXRCF detection + characteristic WENO, in place, with the reference's in-order
 * semantics (weno.rs:90,263).  *troubled (may be NULL) receives the number of limited cells. */
int32_t dgm_apply_limiter(dgm_ctx* ctx, double* solutions, int64_t* troubled);

/* TemperalDisc::compute_time_step(&self, solutions) -> f64 (src/temporal_disc.rs:58). */
int32_t dgm_compute_time_step(dgm_ctx* ctx, const double* solutions, double* time_step);

/* TemperalDisc::rk3(&mut self, spatial_disc, residuals, solutions, time_step)
 * (src/temporal_disc/rk3.rs:7).  One SSP-RK3 step of size time_step with the limiter after
 * each stage; on return solutions holds U^{n+1} and residuals the third stage's residual. */
int32_t dgm_rk3(dgm_ctx* ctx, double* residuals, double* solutions, double time_step);

/* TemperalDisc::time_march(&mut self, spatial_disc, residuals, solutions)
 * (src/temporal_disc.rs:21): while current_step < final_step && current_time < final_time
 * { dt = compute_time_step; clamp to final_time; rk3; advance }.  The loop runs on the device
 * (CUDA graphs, no host round trip per step); the context keeps current_time/current_step
 * across calls like TemperalDisc does. */
int32_t dgm_time_march(dgm_ctx* ctx, double* residuals, double* solutions);

/* TemperalDisc::current_time / current_step (temporal_disc.rs:10-11). */
int32_t dgm_get_clock(dgm_ctx* ctx, double* current_time, int64_t* current_step);
int32_t dgm_set_clock(dgm_ctx* ctx, double current_time, int64_t current_step);

/* SolverParameters::final_time / final_step (solver.rs:12-13): the loop bounds used by
 * dgm_time_march and dgm_advance from the next call on. */
int32_t dgm_set_limits(dgm_ctx* ctx, double final_time, int64_t final_step);

/* ---- device-resident fast path (no host copies of the state per step) ------------------- */

/* Copy a host state ([element][variable][basis]) into the context's resident state, or back. */
int32_t dgm_upload_solutions(dgm_ctx* ctx, const double* solutions);
int32_t dgm_download_solutions(dgm_ctx* ctx, double* solutions);

/* Run up to n_steps steps of time_march on the resident state (stops early at final_step /
 * final_time, as the reference loop does).  Asynchronous: returns after enqueueing; the
 * status of the steps is reported by dgm_synchronize. */
int32_t dgm_advance(dgm_ctx* ctx, int64_t n_steps);

/* Wait for the context's stream; returns the first device-side status raised since the last
 * synchronize (DGM_OK if none). */
int32_t dgm_synchronize(dgm_ctx* ctx);

/* Non-blocking dgm_synchronize: DGM_NOT_READY while work enqueued on the context's stream is
 * still running, otherwise what dgm_synchronize returns.  No counterpart in the reference; used
 * by schedulers that poll many contexts. */
int32_t dgm_query(dgm_ctx* ctx);

/* The context's CUDA stream (cudaStream_t as void*), for callers that order their own work
 * (copies, events) against the solver. */
void* dgm_stream(dgm_ctx* ctx);

/* Diagnostics for per-kernel timing: enqueue one phase of the step on the resident state (phase 0
 * time step, 1 edge flux, 2 element update (stage-2 form, writes the second stage buffer), 3
 * limiter on that buffer: the KXRCF detection launch and the WENO wave launch).  Callers time it
 * with events on dgm_stream().  No counterpart in the reference (it has no kernels). */
int32_t dgm_launch_phase(dgm_ctx* ctx, int32_t phase);
/* Launch configuration of the edge pass (threads per block; blocks, 0 = one thread per
 * (edge slot, Gauss point), else a grid-stride grid of that many blocks) and of the element pass
 * (threads per block = 4 x elements per block).  Threads: multiples of 32 up to 256.  Results do
 * not depend on it.  No counterpart in the reference. */
int32_t dgm_set_launch_config(dgm_ctx* ctx, int32_t edge_threads, int32_t edge_blocks, int32_t element_threads);
int32_t dgm_get_launch_config(dgm_ctx* ctx, int32_t* config /* [3] as above */);
/* Autotuner: times each candidate configuration of the edge pass (every form) and the element
 * pass, and the limiter's detector forms, schedules and wave-kernel grids, on the resident state
 * (repeats launches each, CUDA events) and keeps the fastest; best_us (may be NULL) receives the
 * chosen edge and element times in microseconds.  Call after a state is uploaded. */
int32_t dgm_autotune(dgm_ctx* ctx, int32_t repeats, double* best_us /* [2] */);
/* The edge pass's form (same arithmetic, bitwise identical results): 0 one thread per (edge slot,
 * Gauss point), 1 two lanes per slot, one per side, each loading its element once and evaluating
 * the traces at every point (fewer loads per slot), 2 one lane per (slot, point) with the warp's
 * slots' element records first copied to shared memory by coalesced loads (each record loaded
 * once per slot, all lanes busy; 128-thread blocks whatever the launch configuration says), 3 form 0
 * compiled for 4 blocks of 256 threads per SM (64 registers) instead of 3.
 * No counterpart in the reference. */
int32_t dgm_set_edge_variant(dgm_ctx* ctx, int32_t pair);
int32_t dgm_get_edge_variant(dgm_ctx* ctx);

/* The Navier-Stokes residual (BR2 lifting) in place of the Euler one -- the reference's
 * integrate_over_cell_ns / integrate_over_edges_ns / apply_bc_ns (src/spatial_disc.rs:70-160,
 * 212-348, src/spatial_disc/boundary_condition.rs:121-413, src/spatial_disc/viscous.rs:6-64), which
 * its compute_residuals keeps commented out (src/spatial_disc.rs:34-36) -- for every entry point
 * that evaluates residuals (compute_residuals, rk3, time_march, advance).  FlowParameters::
 * prandtl_number and gas_constant (parameters.json: 0.72, 287) and the reference-space first
 * derivatives of the modes at the edge points, dphi_edge_ref[3][n_edge_gp][n_basis][2] (d/dxi,
 * d/deta: the (1,0) and (0,1) keys of DubinerBasis::dphis_edge_gps, basis_function.rs:152-193).
 * FP64 contexts only (precision 0), not mixed batches: DGM_BAD_ARG otherwise.  enable = 0 returns
 * to the Euler residual.  Adds one launch per stage (the global lifts). */
int32_t dgm_set_viscous(dgm_ctx* ctx, int32_t enable, double prandtl_number, double gas_constant,
                        const double* dphi_edge_ref);
int32_t dgm_get_viscous(dgm_ctx* ctx);
/* The form of the limiter's detection launch (modified_kxrcf, weno.rs:7-85, on every element, one
 * lane each; same arithmetic in both): 0 compact (walks the faces in turn: fewer registers, more
 * lanes in flight), 1 staged (all loads of a round issued together: fewer memory round trips,
 * more registers).  The flags and results are the same.  No counterpart in the reference. */
int32_t dgm_set_limiter_variant(dgm_ctx* ctx, int32_t staged);
/* Current form, and the limiter times the last dgm_autotune measured for forms 0 and 1 at their
 * faster schedule (us; either pointer may be NULL). */
int32_t dgm_get_limiter_variant(dgm_ctx* ctx, int32_t* staged, double* tuned_us /* [2] */);
/* The grid of the limiter's cooperative wave kernel: 0 every co-resident block (the most warps
 * for the reconstructions), 1 one block per SM (fewer arrivals at each grid barrier: cheaper
 * waves when a wave holds few cells).  Same results.  The autotuner picks one.  No counterpart in
 * the reference. */
int32_t dgm_set_limiter_grid(dgm_ctx* ctx, int32_t one_per_sm);
int32_t dgm_get_limiter_grid(dgm_ctx* ctx);
/* The schedule of the limiter's wave launch from wave 2 on (same results bit for bit): 0 barrier
 * (each wave scans the elements still waiting for a lower-index neighbour, passes a grid barrier,
 * then reconstructs the troubled elements it enlisted), 1 queue (warps that have finished the scan
 * already reconstruct enlisted elements while others still scan; no barrier between the two halves
 * of a wave).  Wave 1's cells, enlisted by the detection launch, are reconstructed first in both.
 * No counterpart in the reference. */
int32_t dgm_set_limiter_schedule(dgm_ctx* ctx, int32_t queue);
/* Current schedule, and the best limiter times the last dgm_autotune measured with schedules 0
 * and 1 (us; either pointer may be NULL). */
int32_t dgm_get_limiter_schedule(dgm_ctx* ctx, int32_t* queue, double* tuned_us /* [2] */);
/* Launches of that kernel, and of all kernels, per time-march step. */
int32_t dgm_phase_launches_per_step(dgm_ctx* ctx, int32_t phase);
int32_t dgm_launches_per_step(dgm_ctx* ctx);

/* ---- batches: many independent meshes advanced by the same launches ------------------------
 * No counterpart in the reference, which solves one mesh per run.  A batch context holds the
 * n meshes as one disconnected union mesh; every launch of the step covers all of them, and
 * each instance keeps its own time step, clock, loop bounds and error status (an instance
 * that stops -- final step/time reached or an error raised -- is left untouched by later
 * steps while the others continue).  All instances share the tables (one polynomial order)
 * and hcr; params[i] supplies instance i's cfl / final_time / final_step, and limiter, device
 * and precision are taken from params[0]. */
dgm_ctx* dgm_create_batch(int32_t n_instances, const dgm_mesh_desc* meshes, const dgm_tables_desc* tables,
                          const dgm_params* params, int32_t* status);
int32_t dgm_instance_count(dgm_ctx* ctx);

/* Slots: a batch whose instances reserve room for larger meshes, so that a finished instance's slot
 * can take a new mesh without a new context (continuous batching: a new solve joins the running
 * launches as soon as a slot is free).  capacity[i] gives instance i's room (each at least its
 * initial mesh's count: elements, internal edges, boundary edges, patches); the room of every
 * instance stays in the union mesh, padding included, and costs device memory like elements of
 * their own.  dgm_instance_replace puts `mesh` (which must fit instance i's capacity) and the loop
 * bounds and CFL number of `params` into slot i: the instance's state is zeroed, its clock, loop
 * bounds and status are reset (set its initial solution next), and the other instances are not
 * touched; the call waits for the context's stream first.  Results of every instance are the same
 * in a slot as in an exact-size batch or alone.  No counterpart in the reference. */
typedef struct dgm_slot_capacity {
  int64_t elements;
  int64_t internal_edges;
  int64_t boundary_edges;
  int64_t patches;
} dgm_slot_capacity;
dgm_ctx* dgm_create_batch_slots(int32_t n_instances, const dgm_mesh_desc* meshes, const dgm_slot_capacity* capacity,
                                const dgm_tables_desc* tables, const dgm_params* params, int32_t* status);
int32_t dgm_instance_replace(dgm_ctx* ctx, int32_t i, const dgm_mesh_desc* mesh, const dgm_params* params);
int32_t dgm_instance_capacity(dgm_ctx* ctx, int32_t i, dgm_slot_capacity* capacity);

/* Mixed batch: instances of different polynomial orders (orders[i] in 1..3) advanced by the same
 * launches -- every kernel of a step is one launch over all instances, each block running its
 * instance's order (one persistent cooperative launch for the limiter's waves).  tables[P - 1]
 * describes order P (only the orders present are read); params, capacity (may be NULL) and the
 * instance numbering are as for dgm_create_batch_slots.  Precision 0, 1 or 4 (no tensor cores).  The
 * dgm_instance_*, dgm_advance*, dgm_synchronize, dgm_query, dgm_diagnostics, dgm_limiter_stats and
 * dgm_device_bytes calls work on it; the single-mesh entry points and the launch-configuration
 * calls return DGM_BAD_ARG.  Every instance's results are bitwise those of its order's batch.  No
 * counterpart in the reference. */
dgm_ctx* dgm_create_mixed(int32_t n_instances, const dgm_mesh_desc* meshes, const int32_t* orders,
                          const dgm_tables_desc* tables /* [3] */, const dgm_params* params,
                          const dgm_slot_capacity* capacity, int32_t* status);
/* State of instance i in the reference layout, host <-> device-resident state. */
int32_t dgm_instance_upload(dgm_ctx* ctx, int32_t i, const double* solutions);
int32_t dgm_instance_download(dgm_ctx* ctx, int32_t i, double* solutions);
/* The last residual written by dgm_advance_with_residual / dgm_time_march for instance i. */
int32_t dgm_instance_download_residual(dgm_ctx* ctx, int32_t i, double* residuals);
/* Clock and status of instance i as of the last dgm_synchronize. */
int32_t dgm_instance_state(dgm_ctx* ctx, int32_t i, double* current_time, int64_t* current_step,
                           int32_t* status, int64_t* error_location);
/* Reset instance i's clock, loop bounds and status (applied at the next advance). */
int32_t dgm_instance_set(dgm_ctx* ctx, int32_t i, double current_time, int64_t current_step,
                         double final_time, int64_t final_step);
/* Solver::set_initial_solution (solver.rs:45-79) on the device: the uniform state of
 * InitialSolution (density, angle of attack in degrees, Mach number, pressure; the reference's
 * expressions) projected onto the basis of every element, written to the resident state --
 * bit-identical to the reference's loop.  dgm_set_initial_solution sets every instance,
 * dgm_instance_set_initial instance i only.  The clock is not touched. */
int32_t dgm_set_initial_solution(dgm_ctx* ctx, double density, double angle_of_attack, double mach_number,
                                 double pressure);
int32_t dgm_instance_set_initial(dgm_ctx* ctx, int32_t i, double density, double angle_of_attack,
                                 double mach_number, double pressure);
/* As dgm_advance, additionally writing each step's third-stage residual (for residual norms). */
int32_t dgm_advance_with_residual(dgm_ctx* ctx, int64_t n_steps);

/* FP64 diagnostics of every instance (deterministic reductions), out[8 * i + k]:
 * k = 0..3 integrals of rho, rho u, rho v, rho E over the mesh; 4, 5 pressure force (Fx, Fy)
 * on the wall patches (the force on the body); 6 sum of squares of the density residual's
 * modal coefficients of the last residual written (0 unless use_residual); 7 element count.
 * No counterpart in the reference (it computes no forces or norms). */
int32_t dgm_diagnostics(dgm_ctx* ctx, int32_t use_residual, double* out);
/* The same diagnostics without waiting: dgm_enqueue_diagnostics enqueues their computation after
 * the work already on the context's stream, with a copy into a pinned host buffer of the context;
 * dgm_collected_diagnostics waits for that copy (not for later work) and returns it in out (as
 * above; DGM_BAD_ARG before the first enqueue).  A serving loop enqueues them behind each chunk of
 * steps and reads them when the chunk is done, with no device work on its check path.  Not for
 * mixed batches. */
int32_t dgm_enqueue_diagnostics(dgm_ctx* ctx, int32_t use_residual);
int32_t dgm_collected_diagnostics(dgm_ctx* ctx, double* out);

/* Cell fields of write_to_vtk (src/io/write_results.rs:33-61) for instance i of the resident
 * state: fields[e][0..4] = density, x velocity, y velocity, pressure from each element's mode-0
 * coefficients, computed on the device in FP64 with the reference's expressions (bit-identical
 * to them).  The host writes the file (dgm_in_rust_b200.output.write_to_vtk). */
int32_t dgm_cell_fields(dgm_ctx* ctx, int32_t instance, double* fields /* [ne][4] */);
/* The context's precision mode (dgm_params::precision). */
int32_t dgm_precision(dgm_ctx* ctx);

/* Edge (HLLC failures) or element (limiter failures) index flagged by the last error. */
int64_t dgm_error_location(dgm_ctx* ctx);

/* Limited cells and limiter waves of the most recent limiter pass (diagnostics). */
int32_t dgm_limiter_stats(dgm_ctx* ctx, int64_t* troubled, int32_t* waves);

/* Bytes of device memory held by the context. */
int64_t dgm_device_bytes(dgm_ctx* ctx);

const char* dgm_status_string(int32_t status);

/* ---- allocation-free variant ------------------------------------------------------------ */

/* The CFL time step -- the minimum over the elements of cfl * h_min / (|u| + c), with the state of
 * each element taken as the sum of its modal coefficients -- for callers that cannot allocate
 * device memory: hosts whose device memory belongs to another allocator, code running while a
 * stream is captured into a CUDA graph, real-time loops.  It needs no dgm_ctx and calls no
 * cudaMalloc/cudaFree: the caller passes device pointers to the state in the layout
 * [n_elements][4][n_basis] and to the element minimum heights [n_elements], and a device double
 * that receives the time step (1e10 when no element gives a smaller finite value); the work is
 * enqueued on `stream` (cudaStream_t, NULL = default).  cfl must be > 0 and hcr > 1, else
 * DGM_BAD_ARG.  Scratch is a fixed 32 KiB array in the library image (every GPU that loads the
 * library holds it until exit) of 4096 per-block minima, which caps n_elements at 8,388,608:
 * larger sizes return DGM_BAD_ARG without launching anything.  Every used scratch slot is
 * rewritten by every call; calls that overlap on the GPU (other streams, other host threads) share
 * the array and race.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current and keeps it for the life of the process: make
 * that first call before any stream capture, and make no call after a cudaDeviceReset of a device
 * already used (the kept address is then stale).  A CUDA error left pending by earlier work is
 * returned as DGM_CUDA_ERROR before anything is launched and stays pending.  This entry point has
 * no counterpart in the reference, which allocates freely. */
int32_t dgm_compute_time_step_noalloc(const double* solutions, const double* minimum_height,
                                      int64_t n_elements, int32_t n_basis, double cfl, double hcr,
                                      double* time_step, void* stream);

/* Library version string. */
const char* dgm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DGM_B200_H */
