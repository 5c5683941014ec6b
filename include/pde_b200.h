/*
 * pde_b200.h -- C ABI of the B200 (sm_100a) finite-difference hot path.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (passed as void*, i.e. a cudaStream_t; NULL = legacy default stream) and
 * returns PDE_OK (0) or a negative PDE_ERR_* code.  Nothing aborts, nothing
 * allocates device memory inside an operator call: scratch buffers and
 * outputs are owned by the caller.
 *
 * Data layout (identical to PDE_Module's Warp `array3d(dtype=vec(N)/mat(N,D))`):
 *   fp32, C-contiguous, shape (X, Y, Z, N) or (X, Y, Z, N, D); X, Y, Z include
 *   the ghost layers; an axis of size 1 is not a spatial dimension (a 2D grid
 *   is (X, Y, 1, ...)).  "Eligible" axes are those with size > 1, listed in
 *   ascending order; D is their count.  Interior ("stencil") cells are the
 *   indices [g, n-g) on every eligible axis (boundary nodes sit at g and n-g-1).
 *
 * Reference interfaces replaced (paths relative to the PDE_Module project):
 *   pde_laplacian   FDM/functional/_laplacian.py:5-36 + FDM/kernel/laplacian.py:34-59
 *   pde_grad        FDM/functional/_grad.py:5-36 + FDM/kernel/grad.py:37-102
 *   pde_divergence  FDM/functional/_divergence.py:4-24 + FDM/kernel/divergence.py:32-106
 *   pde_euler       time_step/forwardEuler.py:41-81
 *   pde_bc_apply    FDM/boundary/functional_boundary.py:260-294 (copy + group launches)
 *                   with the kernel of functional_boundary.py:312-402 and the value
 *                   functions of FDM/boundary/boundary_functions.py:9-92
 */
#ifndef PDE_B200_H
#define PDE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PDE_OK                 0
#define PDE_ERR_ARG          (-1)  /* null pointer / bad enum / bad count          */
#define PDE_ERR_SHAPE        (-2)  /* shape inconsistent with the operator         */
#define PDE_ERR_GHOST        (-3)  /* ghost width smaller than the stencil radius  */
#define PDE_ERR_ALIGN        (-4)  /* pointer alignment requirement not met        */
#define PDE_ERR_CUDA         (-5)  /* a CUDA runtime call failed                   */
#define PDE_ERR_UNSUPPORTED  (-6)  /* valid request this build does not implement  */
#define PDE_ERR_TIMEOUT      (-7)  /* a bounded device-side wait gave up           */
#define PDE_ERR_TOO_LARGE    (-8)  /* size above a documented maximum              */

/* Boundary-condition kinds: values of FDM/boundary/flags.py:8-16. */
#define PDE_BC_DIRICHLET     1
#define PDE_BC_VON_NEUMANN   2
/* Boundary value functions: boundary_functions.py:9-47 (constant), :51-92 (ramp). */
#define PDE_BC_FUNC_CONSTANT 0
#define PDE_BC_FUNC_RAMP     1

/* Face bits for standard boundary groups (functional_boundary.py:111-137). */
#define PDE_FACE_XM  (1 << 0)  /* "-X" */
#define PDE_FACE_XP  (1 << 1)  /* "+X" */
#define PDE_FACE_YM  (1 << 2)  /* "-Y" */
#define PDE_FACE_YP  (1 << 3)  /* "+Y" */
#define PDE_FACE_ZM  (1 << 4)  /* "-Z" */
#define PDE_FACE_ZP  (1 << 5)  /* "+Z" */

/* Largest number of components a fused (boundary-in-the-stencil) kernel takes. */
#define PDE_FUSED_MAX_COMP   4
/* Largest number of boundary groups a compiled rule table holds. */
#define PDE_MAX_GROUPS       16

/* Uniform grid: array shape including ghosts, ghost width, stencil order, spacing.
 * Stencil weights are formed on the host in double from dx and rounded to fp32,
 * as the reference forms them (FDM/module/laplacian.py:33-35, grad.py:37-39,
 * divergence.py:37-39):
 *   Laplacian order 2: ( 1, -2,  1)/dx^2        order 4: (-1, 16, -30, 16, -1)/(12 dx^2)
 *   first derivative order 2: (-1, 0, 1)/(2 dx) order 4: ( 1, -8,   0,  8, -1)/(12 dx)
 * Order 4 has no reference counterpart (the reference rejects custom stencils). */
typedef struct PdeGrid {
  int64_t shape[3];     /* X, Y, Z including ghost layers                        */
  int32_t ghost_cells;  /* g; must be >= order/2                                 */
  int32_t order;        /* 2 or 4                                                */
  double  dx;           /* grid spacing                                          */
} PdeGrid;

/* One boundary group (a FunctionBC of functional_boundary.py:25-55). */
typedef struct PdeBCGroup {
  const int32_t* node_ids;  /* device pointer: flat C-order node ids (X*Y*Z index) */
  int32_t  count;           /* number of node ids                                  */
  int32_t  type;            /* PDE_BC_DIRICHLET or PDE_BC_VON_NEUMANN              */
  uint32_t comp_mask;       /* bit v set <=> component v is set (output_ids)       */
  int32_t  func;            /* PDE_BC_FUNC_CONSTANT or PDE_BC_FUNC_RAMP            */
  float    value;           /* constant (or ramp target)                           */
  float    t_max;           /* ramp time scale (ramp only)                          */
  int32_t  face_mask;       /* PDE_FACE_* bits when the group is a standard face
                               group ("ALL" = every eligible face); 0 = custom ids */
} PdeBCGroup;

/* Boundary groups compiled for the fused kernels: for each node class (per
 * axis: low node / other / high node, index kx*9+ky*3+kz) the group whose write
 * wins at the node and at each adjacent ghost, per component; -1 = none.   */
typedef struct PdeBCGroupParam {
  int32_t  type;
  uint32_t comp_mask;
  int32_t  func;
  float    value;
  float    t_max;
} PdeBCGroupParam;

typedef struct PdeBCRules {
  int32_t ncomp;
  int32_t ngroups;
  float   dx32;                               /* fp32 dx (ExplicitUniformGridStencil.py:27) */
  int32_t has_ramp;                           /* any group uses a time-dependent value       */
  PdeBCGroupParam group[PDE_MAX_GROUPS];
  int8_t  node_group[27];                     /* last Dirichlet group containing the node    */
  int8_t  ghost_group[27][3][PDE_FUSED_MAX_COMP]; /* last group setting ghost comp       */
  int8_t  pad[1];
} PdeBCRules;

/* ---- library --------------------------------------------------------- */
int         pde_version(void);
const char* pde_strerror(int status);
/* Reads and clears the device-side error word (bounded waits that gave up,
 * bounds checks that failed).  0 = none.  Synchronises the given stream. */
int         pde_device_error(void* stream);

/* Bound of every device-side wait of the library (the stream3d kernels'
 * mbarrier waits, the batched rollout's tile-progress waits): a wait that runs
 * this long gives up, records PDE_ERR_TIMEOUT in the error word and lets its
 * kernel return; once the word is set, every other wait gives up at once.
 * ns = 0 restores the default (2 s).  Process-wide, read at each launch;
 * returns the previous bound.  No counterpart in the reference (Warp kernels
 * do not wait on one another). */
#define PDE_WAIT_LIMIT_DEFAULT_NS 2000000000ull
uint64_t    pde_set_wait_limit_ns(uint64_t ns);

/* Test hook of the bounded wait: one thread waits until *word >= target (word:
 * a device uint32) with the progress-wait code of the batched rollout, under
 * the current bound, and records PDE_ERR_TIMEOUT if it gives up.  No
 * counterpart in the reference. */
int         pde_wait_probe(const uint32_t* word, uint32_t target, void* stream);

/* Kernel selection for pde_laplacian/pde_grad/pde_divergence: PDE_DISPATCH_AUTO
 * picks the TMA streaming kernels where they apply, PDE_DISPATCH_GENERIC forces
 * the general kernels (same arithmetic, used to cross-check the two bitwise).
 * Process-wide; returns the previous mode. */
#define PDE_DISPATCH_AUTO    0
#define PDE_DISPATCH_GENERIC 1
int         pde_set_dispatch(int mode);

/* Tile configuration of the 3D streaming kernel used for one operator and
 * order: candidate 0 (default) .. 3; op is PDE_OP_*, ncomp_in the input's
 * component count (Laplacian 1 or 3, Grad 1, Divergence 3).  Candidates above
 * 0 apply to exact mode on grids with even Y and Z (others keep candidate 0).  candidate -1 queries.  Process-wide; returns the
 * previous candidate or a negative status.  The tuner in
 * pde_module_b200/tuning.py sweeps these. */
#define PDE_OP_LAPLACIAN  0
#define PDE_OP_GRAD       1
#define PDE_OP_DIVERGENCE 2
int         pde_stream3d_select(int32_t op, int32_t order, int32_t ncomp_in, int32_t candidate);

/* ---- operators (one launch each; out must not alias in) ------------- */

/* out[c] = alpha * sum_{axis} sum_{tap} w[tap] * in[c + shift*e_axis], per component,
 * for every interior cell c; ghost cells of out are not written.
 * in/out: (X,Y,Z,ncomp).  Summation order: axes ascending, taps low to high,
 * alpha last, every product and sum rounded separately (FDM/kernel/laplacian.py:34-46). */
int pde_laplacian(const float* in, float* out, const PdeGrid* grid, int32_t ncomp,
                  float alpha, void* stream);

/* out[c][n][a] = alpha * sum_tap w[tap] * in[c + shift*e_axis(a)][n]
 * in: (X,Y,Z,ncomp)  out: (X,Y,Z,ncomp,D)  (ncomp==1: the vec(D) output of Grad).
 * FDM/kernel/grad.py:78-100. */
int pde_grad(const float* in, float* out, const PdeGrid* grid, int32_t ncomp,
             float alpha, void* stream);

/* out[c][n] = alpha * sum_a sum_tap w[tap] * in[c + shift*e_axis(a)][n][a]
 * in: (X,Y,Z,nrows,D) (nrows==1: vec(D) input)  out: (X,Y,Z,nrows).
 * FDM/kernel/divergence.py:85-106.  One launch (the reference launches twice,
 * FDM/module/divergence.py:98-110, with an identical result). */
int pde_divergence(const float* in, float* out, const PdeGrid* grid, int32_t nrows,
                   float alpha, void* stream);

/* Arithmetic modes of the _ex operator variants.  PDE_MODE_EXACT (what the
 * plain entry points use) rounds every product and sum of the reference's sum
 * separately, in its order: results are bit-identical to the reference
 * algorithm.  PDE_MODE_FAST sums taps that share a weight before multiplying,
 * folds alpha into the weights and uses FMA (3D streaming kernels; other
 * shapes run the exact kernels).  Its results differ from exact ones by a few
 * float32 roundings of the summed terms (relative L2 difference ~1e-7 on
 * random fields) and a zero-weight tap no longer propagates NaN/Inf. */
#define PDE_MODE_EXACT 0
#define PDE_MODE_FAST  1
int pde_laplacian_ex(const float* in, float* out, const PdeGrid* grid, int32_t ncomp, float alpha,
                     int32_t mode, void* stream);
int pde_grad_ex(const float* in, float* out, const PdeGrid* grid, int32_t ncomp, float alpha, int32_t mode,
                void* stream);
int pde_divergence_ex(const float* in, float* out, const PdeGrid* grid, int32_t nrows, float alpha,
                      int32_t mode, void* stream);

/* out[i] = y[i] + dt * k[i] for i < count (floats), time_step/forwardEuler.py:70-79. */
int pde_euler(const float* y, const float* k, float dt, float* out, int64_t count,
              void* stream);

/* out = copy(in); then for each group in order: Dirichlet writes the node vector
 * (input vector with the set components replaced by the value) and, for every
 * eligible axis on which the node sits at index g or n-g-1, the ghost one step
 * outside: ghost[v] = 2*val - in[adj][v]; Von Neumann writes only the ghost:
 * ghost[v] = -sign(inc)*2*dx*val + in[adj][v].  t_device: device pointer to one
 * float (time, ramp functions only; may be NULL when no group is a ramp).
 * functional_boundary.py:260-294, 357-400. */
int pde_bc_apply(const float* in, float* out, const PdeGrid* grid, int32_t ncomp,
                 const PdeBCGroup* groups, int32_t ngroups, const float* t_device,
                 void* stream);

/* NEW (no reference counterpart: flags.py has no periodic kind).  In place:
 * every ghost cell along the axes in axis_mask (bit a = axis a) takes the value
 * of the interior cell congruent to it modulo the interior extent; axes are
 * filled in ascending order over the full extent of the other axes, so edge and
 * corner ghosts are filled too. */
int pde_periodic_fill(float* u, const PdeGrid* grid, int32_t ncomp, int32_t axis_mask,
                      void* stream);

/* Host-only: compile standard face groups into the rule table the fused kernels
 * read.  Fails with PDE_ERR_UNSUPPORTED when a group has face_mask == 0 (custom
 * node lists) or ncomp > PDE_FUSED_MAX_COMP. */
int pde_bc_compile(const PdeBCGroup* groups, int32_t ngroups, const PdeGrid* grid,
                   int32_t ncomp, PdeBCRules* rules_out);

/* ---- fused explicit steps (boundary fill + Laplacian + forward Euler) ---- */

/* nsteps of   u2 = BC(u);  u <- u2 + dt * (alpha * Laplacian(u2))   on a 2D or 3D
 * grid, the composition of time_step/forwardEuler.py:41-61, FDM/module/laplacian.py
 * and functional_boundary.py (examples/2D_Heat_Equation.py:57-65), bit-identical to
 * running those three operators step by step.  Ghost cells of the result hold the
 * boundary-filled values of the last step (the unfused chain leaves the same values
 * when the Laplacian output's ghost cells are zero).
 * u_in: initial field; u_out: result; work: scratch of the same size (used as the
 * ping-pong buffer when nsteps > steps_per_pass).  u_out may equal u_in.
 * steps_per_pass: temporal-blocking depth k (0 = choose).  2D (Z == 1) grids use
 * shared-memory tiles with k steps per pass.  3D grids whose interior has at
 * least 3 cells per axis stream along X with k steps per pass (k at most 4 for
 * one component, 2 for more; deeper requests run at that depth).  At k = 1 a
 * scalar field whose shape takes the double-row map (even Y and Z, plane pitch
 * a multiple of 4 floats, even g - R) runs a surface fill and the TMA streaming
 * heat step per step, and 0 chooses k = 1 there; otherwise 0 chooses 2 for
 * order 2 and 1 for order 4 (pde_heat_pass_depth).  Smaller 3D grids take one
 * step per pass.  The input is never written (the streaming path copies it once
 * into a buffer of the call unless u_out == u_in).
 * Constant-valued groups only: rules with a ramp group (has_ramp) give
 * PDE_ERR_UNSUPPORTED here; pde_heat_rollout_at takes them. */
int pde_heat_rollout(const float* u_in, float* u_out, float* work, const PdeGrid* grid,
                     int32_t ncomp, const PdeBCRules* rules, float alpha, float dt,
                     int32_t nsteps, int32_t steps_per_pass, void* stream);

/* pde_heat_rollout with time-dependent boundary groups (ramps,
 * boundary_functions.py:77-92, set through functional_boundary.py:237,254-255,
 * where the loop passes t to every call).  Step n (0-based) fills the boundary
 * at t = fp32(t0 + n * t_step), the sum and product taken in double and each
 * rounded on its own, as a Python loop calling BC(u, t0 + n*dt) computes it;
 * the result is bit-identical to that loop of the three operators.  t_step is
 * the time step as a double (the caller's dt before its rounding to fp32).
 * Constant groups behave as in pde_heat_rollout. */
int pde_heat_rollout_at(const float* u_in, float* u_out, float* work, const PdeGrid* grid,
                        int32_t ncomp, const PdeBCRules* rules, float alpha, float dt,
                        int32_t nsteps, int32_t steps_per_pass, double t0, double t_step,
                        void* stream);

/* pde_heat_rollout_at continuing a run at step n0 >= 0: step n of the call
 * fills the boundary at fp32(t0 + (n0 + n) * t_step), so consecutive calls of
 * k steps (n0 = 0, k, 2k, ...) equal one call of the whole run bit for bit (the
 * slab rollout's blocks between halo exchanges).  u_in is scratch here: its
 * contents may be overwritten (the one-step 3D path fills its boundary cells in
 * place instead of copying it first). */
int pde_heat_rollout_from(const float* u_in, float* u_out, float* work, const PdeGrid* grid,
                          int32_t ncomp, const PdeBCRules* rules, float alpha, float dt,
                          int32_t nsteps, int32_t steps_per_pass, double t0, double t_step,
                          int32_t n0, void* stream);

/* Steps per pass pde_heat_rollout uses on this grid for a steps_per_pass
 * request (0 = choose), or a negative status.  Needs no GPU. */
int pde_heat_pass_depth(const PdeGrid* grid, int32_t ncomp, int32_t steps_per_pass);

/* ---- differentiable heat rollout (new: the reference has the forward loop
 * only, examples/2D_Heat_Equation.py:57-65, with a scalar alpha) ----
 * 2D grids, one component, order 2 or 4, constant-valued face groups.
 * Forward step with a per-cell diffusivity field alpha (X, Y):
 *   v = BC(u);  S = Lap(v) (alpha 1);  u' = v + dt*(alpha o S) on stencil cells, v elsewhere
 * (bit-identical to pde_heat_rollout when alpha is constant).  `lstates`, if
 * not NULL, receives S of step n at lstates + n*X*Y for n = 0..nsteps-1 on the
 * stencil cells (other cells unspecified).  `work`: one field of scratch. */
int pde_heat_forward(const float* alpha, const float* u_in, float* u_out, float* work, const PdeGrid* grid,
                     const PdeBCRules* rules, float dt, int32_t nsteps, int32_t steps_per_pass, float* lstates,
                     void* stream);
/* pde_heat_forward with time-dependent groups (ramps, boundary_functions.py:77-92):
 * step n of this call is rollout step n0 + n and fills the boundary at
 * t = fp32(t0 + (n0 + n) * t_step), the sum and product in double, each rounded
 * on its own, as a loop calling BC(u, t0 + k*dt) computes it.  pde_heat_forward
 * refuses ramp groups (PDE_ERR_UNSUPPORTED).  The adjoint takes the same rules:
 * the fill is affine in u, its values enter the forward only. */
int pde_heat_forward_at(const float* alpha, const float* u_in, float* u_out, float* work, const PdeGrid* grid,
                        const PdeBCRules* rules, float dt, int32_t nsteps, int32_t steps_per_pass,
                        float* lstates, double t0, double t_step, int32_t n0, void* stream);
/* Discrete adjoint of nsteps forward steps: lam_in = dJ/du^N, lam_out =
 * dJ/du^0; grad_alpha += dJ/dalpha (accumulated in step order n = N-1..0);
 * lstates as written by pde_heat_forward for the same steps. */
int pde_heat_adjoint(const float* alpha, const float* lam_in, float* lam_out, const float* lstates,
                     float* grad_alpha, const PdeGrid* grid, const PdeBCRules* rules, float dt, int32_t nsteps,
                     int32_t steps_per_pass, float* work, void* stream);

/* ---- fractional-step lid-driven cavity (new: the reference's LDC uses
 * artificial compressibility, examples/LDC/LDC_Graph_Capture.py:71-90) ---- */
typedef struct PdeLDCParams {
  float   nu;               /* kinematic viscosity                              */
  float   dt;               /* time step                                        */
  int32_t jacobi_iters;     /* pressure sweeps per step                         */
  int32_t jacobi_per_pass;  /* sweeps per launch (temporal blocking), 0 = 10    */
} PdeLDCParams;

/* nsteps of the projection method on a 2D grid, u (X,Y,1,2) and p (X,Y,1,1)
 * advanced in place, composed of the reference operators in float32, one
 * rounding per product and sum:
 *   u2 = BC_u(u); u* = u2 + dt*(nu*Lap(u2) - Grad(u2) u2)
 *   rhs = (1/dt)*Div(BC_u(u*))
 *   jacobi_iters times: p <- 0.25*(pW + pE + pS + pN - dx^2*rhs) on BC_p(p)
 *   u = BC_u(u*) + dt*(-Grad(BC_p(p)))
 * u_rules / p_rules: compiled boundary groups (pde_bc_compile) of the velocity
 * (2 components) and pressure (1).  u_star, p_tmp, rhs: scratch of u's, p's and
 * p's size.  resid: device array of nsteps floats (or NULL) receiving the sum of
 * squared pressure updates of each step's last sweep. */
int pde_ldc_rollout(float* u, float* p, float* u_star, float* p_tmp, float* rhs, float* resid,
                    const PdeGrid* grid, const PdeBCRules* u_rules, const PdeBCRules* p_rules,
                    const PdeLDCParams* params, int32_t nsteps, void* stream);
/* pde_ldc_rollout with time-dependent groups (a ramped lid, as the reference's
 * function-BC cavity, Benchmark/Functional_BC/LDC_Graph Function.py:44-113,
 * with boundary_functions.py:77-92): step n (0-based) fills every velocity and
 * pressure boundary of the step at t = fp32(t0 + n * t_step), the sum and
 * product in double, each rounded on its own, as a loop calling the boundaries
 * with that time computes it.  pde_ldc_rollout refuses ramp groups
 * (PDE_ERR_UNSUPPORTED). */
int pde_ldc_rollout_at(float* u, float* p, float* u_star, float* p_tmp, float* rhs, float* resid,
                       const PdeGrid* grid, const PdeBCRules* u_rules, const PdeBCRules* p_rules,
                       const PdeLDCParams* params, int32_t nsteps, double t0, double t_step, void* stream);

/* ---- weakly compressible flow, RK2 (new: the reference composes the step from
 * its modules, examples/LDC/LDC_RK2.py) ----
 * Parameters as the caller's doubles; each is rounded to fp32 as the module
 * chain receives it (dt/2 is formed in double first). */
typedef struct PdeWCParams {
  double nu;    /* viscosity: Lap(u, nu)                      */
  double eps;   /* biharmonic damping: Lap(Lap(u, nu), eps)   */
  double c2;    /* sound speed squared: p = c2 * (rho - rho0) */
  double rho0;  /* reference density                          */
  double dt;    /* time step                                  */
} PdeWCParams;

/* nsteps RK2 (midpoint) steps of momentum m (X,Y,1,2) and density rho (X,Y,1,1),
 * one fused launch per step, bit-identical to the composition of the reference
 * operators (one rounding per product and sum, time_step/rungeKatta.py:123-174):
 *   bc(m, rho) = (rho' * u', rho') with u = m / rho, u' = BC_u(u), rho' = BC_rho(rho)
 *   f(m, rho)  = (((Grad(c2 (rho - rho0), -1) - Div(outer(m, u), 1)) + Lap(u, nu))
 *                 + Lap(Lap(u, nu), eps),  Div(m, -1)),  u = m / rho
 *   y0 = bc(y);  y1 = bc(y0 + (dt/2) f(y0));  y' = y0 + dt f(y1)
 * (operator outputs 0 outside the array interior).  u_rules: 2 components,
 * rho_rules: 1 (pde_bc_compile, constant face groups).  2D grids, order 2.
 * work: 3 X Y floats.  m_out / rho_out may equal the inputs. */
int pde_wc_rk2(const float* m_in, const float* rho_in, float* m_out, float* rho_out,
               const PdeGrid* grid, const PdeBCRules* u_rules, const PdeBCRules* rho_rules,
               const PdeWCParams* params, int32_t nsteps, float* work, void* stream);

/* One phase of a fractional step on a slab of the cavity: the rows
 * [x_offset, x_offset + grid->shape[0]) of a domain of x_global rows (grid
 * describes the slab's arrays; the other extents, ghost cells and dx are the
 * domain's).  Results are written on the owned rows [own_lo, own_hi) only; rows
 * beyond them are halo rows a host fills from the neighbouring slabs between
 * phases (pde_module_b200.distributed).  Halo rows needed on a cut side
 * (own_lo > 0, own_hi < x_global): 1 for PREDICT, DIVERGENCE (u_star) and
 * PROJECT (u_star, p_in); nsweeps + 1 for JACOBI (p_in and rhs), which runs
 * nsweeps sweeps from p_in into p_out (distinct) and, when `last` is set and
 * resid is not NULL, adds the sum of squared updates of its owned cells to *resid.
 * With one slab holding every row the phases compose pde_ldc_rollout's step,
 * bit for bit. */
typedef struct PdeSlab {
  int64_t x_global;   /* rows of the whole domain, ghosts included          */
  int64_t x_offset;   /* global row of the arrays' first row                */
  int64_t own_lo;     /* first owned global row                             */
  int64_t own_hi;     /* one past the last owned global row                 */
} PdeSlab;
#define PDE_LDC_PREDICT    0
#define PDE_LDC_DIVERGENCE 1
#define PDE_LDC_JACOBI     2
#define PDE_LDC_PROJECT    3
int pde_ldc_slab_step(int32_t phase, float* u, float* u_star, const float* p_in, float* p_out, float* rhs,
                      float* resid, const PdeGrid* grid, const PdeSlab* slab, const PdeBCRules* u_rules,
                      const PdeBCRules* p_rules, const PdeLDCParams* params, int32_t nsweeps, int32_t last,
                      void* stream);

/* ---- differentiable 2D wave equation (new; the reference's wave examples step a
 * first-order (u, v) pair with forward Euler, tests/FDM/test_WaveStanding.py:71-76) ----
 * State on the cells strictly inside the Dirichlet node ring (nodes and ghosts 0),
 * K = dt^2 c^2 a field, L the 5-point Laplacian in the reference's order:
 *   u^{n+1} = 2 u^n - u^{n-1} + K o L(u^n) + src[n] at src_cell
 * pde_wave_forward: nsteps from (u^{n0-1}, u^{n0}) = (u_prev, u_cur) to
 * (out_prev, out_cur) = (u^{n0+nsteps-1}, u^{n0+nsteps}); src_cell < 0: no source.
 * lstates (NULL or nsteps fields): lstates[j] = L(u^{n0+j}) on the cells inside
 * the node ring, 0 elsewhere (the Laplacian each step forms).  work: 2 fields.
 * steps_per_pass: temporal-blocking depth (0 = 8). */
int pde_wave_forward(const float* K, const float* u_prev, const float* u_cur, float* out_prev, float* out_cur,
                     const float* src, int64_t src_cell, int32_t n0, int32_t nsteps, int32_t steps_per_pass,
                     float* lstates, float* work, const PdeGrid* grid, void* stream);
/* Discrete adjoint over steps n = nsteps-1 .. 0 of a segment whose forward wrote
 * lstates[j] = L(u^j) (j = 0 .. nsteps-1):  mu^n = 2 mu^{n+1} - mu^{n+2} + L(K o mu^{n+1}),
 * grad_K += mu^{n+1} o L(u^n) (one add per cell and step, n descending).
 * In: (mu_next, mu_next2) = (mu^{nsteps}, mu^{nsteps+1}); out: (mu_out, mu_out_next) =
 * (mu^0, mu^1).  work: 2 fields. */
int pde_wave_adjoint(const float* K, const float* mu_next, const float* mu_next2, float* mu_out,
                     float* mu_out_next, const float* lstates, float* grad_K, int32_t nsteps,
                     int32_t steps_per_pass, float* work, const PdeGrid* grid, void* stream);
/* pde_wave_forward (nsteps_fwd steps from n0, L(u^n) stored to lstates_fwd; the
 * final state is not returned) and pde_wave_adjoint (nsteps_adj steps from
 * lstates_adj, grad_K accumulated) of two different segments in one sequence of
 * paired launches: each launch advances every tile through up to
 * steps_per_pass steps of both, so the two interleave on each SM.  Results are
 * bit-identical to the two calls made separately.  Either step count may be 0
 * (that part's pointers may then be NULL).  The pass depth is steps_per_pass or
 * the deepest below it whose shared-memory region fits.  work: 6 fields. */
int pde_wave_pair(const float* K, const float* u_prev, const float* u_cur, int32_t n0, int32_t nsteps_fwd,
                  float* lstates_fwd, const float* mu_next, const float* mu_next2, float* mu_out, float* mu_out_next,
                  const float* lstates_adj, float* grad_K, int32_t nsteps_adj, const float* src, int64_t src_cell,
                  int32_t steps_per_pass, float* work, const PdeGrid* grid, void* stream);
/* Launch shape of the tiled 2D kernels of pde_heat_rollout[_at],
 * pde_heat_forward, pde_heat_adjoint, pde_wave_forward, pde_wave_adjoint,
 * pde_wave_pair, pde_wc_rk2 and the Jacobi sweeps of pde_ldc_rollout and
 * pde_ldc_slab_step, process-wide:
 * output tile (sides 8..256; (0, 0) = automatic: the largest of 32x64, 32x32,
 * 16x32 that gives every SM a tile, enlarged slightly when the count is just
 * above a multiple of the SM count; for the fused heat rollout square tiles of
 * about one per SM, sides 16..64) and threads per block (256, 512, 1024;
 * 0 = automatic: for the wave and differentiable-heat kernels 1024 with up to one
 * tile per SM, 512 up to two, else 256; 512 for the fused heat rollout and the
 * weakly compressible step (which takes 256 or 512); 256 for the Jacobi sweeps).
 * The Jacobi sweeps with both left automatic take one near-square tile per SM
 * and 1024 threads when those tiles have sides of at least 32 and their region
 * holds at most 12 cells per thread.  Any shape whose region holds at most 12
 * cells per thread runs the register cell-list Jacobi kernel, others the
 * flat-walk kernel (same results). */
int pde_set_launch_2d(int32_t tile_x, int32_t tile_y, int32_t threads);

/* Launch shape of the 3D streaming heat rollout (pde_heat_rollout[_at] on 3D
 * grids): largest tile sides along Y and Z (capped at the compiled maxima, 32
 * for one component) and the number of chunks the X axis is split into
 * (items = tiles x chunks on a persistent grid); 0 = chosen per launch.
 * Process-wide; for tuning.  Results do not depend on it.  No counterpart in
 * the reference (its kernels are launched by Warp). */
int pde_set_launch_3d(int32_t tile_y, int32_t tile_z, int32_t chunks);

/* ---- batched rollouts (new: the reference advances every grid with its own
 * module chain, examples/2D_Heat_Equation.py:57-65, three launches per step
 * per grid).  Many independent 2D grids of uneven sizes advance together in
 * ONE persistent launch over a tile work queue: items (time block, grid, tile)
 * in time-block-major order; a tile starts a time block once its 3x3
 * neighbours finished the previous one (bounded waits, PDE_ERR_TIMEOUT).
 * Heat results are bit-identical to pde_heat_rollout per grid; wave results to
 * pde_wave_forward with a constant K field and no source. ---- */
#define PDE_BATCH_HEAT 0
#define PDE_BATCH_WAVE 1

typedef struct PdeBatchGrid {
  float*  field;       /* heat: u; wave: u^n.  (X, Y, 1, 1) float32 incl. ghosts,
                          overwritten by the result (u after nsteps; u^{n+nsteps}) */
  float*  field_prev;  /* wave: u^{n-1}, overwritten by u^{n+nsteps-1}; heat: NULL  */
  float*  scratch;     /* device scratch: X*Y floats (heat), 2*X*Y floats (wave)    */
  int64_t shape[2];    /* X, Y including ghosts                                     */
  double  dx;          /* spacing (Laplacian weights; heat Neumann ghosts)          */
  float   coef;        /* heat: diffusivity alpha; wave: K = dt^2 c^2               */
  float   dt;          /* heat: time step; wave: unused                             */
} PdeBatchGrid;

typedef struct PdeBatchPlan {
  void*      table;           /* device: descriptors + queue state (in `work`)      */
  int32_t    kind;            /* PDE_BATCH_HEAT or PDE_BATCH_WAVE                   */
  int32_t    ngrids;
  int32_t    total_tiles;
  int32_t    ghost_cells;
  int32_t    order;           /* heat: 2 or 4; wave: 2                              */
  int32_t    tile_x, tile_y;  /* output tile (cells, ghosts included)               */
  int32_t    steps_per_pass;  /* time-block depth k                                 */
  int32_t    blocks;          /* persistent grid size                               */
  int32_t    smem_bytes;
  PdeBCRules rules;           /* heat: the boundary groups every grid shares        */
} PdeBatchPlan;

/* Device bytes `work` must hold for these grids and tile (0 = default). */
int pde_batch_work_bytes(const PdeBatchGrid* grids, int32_t ngrids, int32_t tile_x, int32_t tile_y,
                         uint64_t* bytes);
/* Validate the grids, choose the launch (tile 0 = 32 x 64, steps_per_pass 0 =
 * 8) and upload the descriptor table into `work` on `stream` (from pageable
 * host memory: call it outside stream capture).  `rules` (heat only; compiled
 * by pde_bc_compile for any grid of the batch, ncomp 1, constant values) is
 * copied into the plan; each grid's own dx is used for its Neumann ghosts.
 * The halo (heat k*R+1, wave k) may not exceed a tile side. */
int pde_batch_plan(int32_t kind, const PdeBatchGrid* grids, int32_t ngrids, int32_t ghost_cells, int32_t order,
                   const PdeBCRules* rules, int32_t tile_x, int32_t tile_y, int32_t steps_per_pass, void* work,
                   uint64_t work_bytes, PdeBatchPlan* plan, void* stream);
/* Advance every grid of the plan nsteps: one memset of the queue state and one
 * kernel launch, so it can be captured in a CUDA graph. */
int pde_batch_rollout(const PdeBatchPlan* plan, int32_t nsteps, void* stream);
/* pde_batch_rollout for heat plans whose groups include ramps
 * (boundary_functions.py:77-92): step n (0-based) of grid i fills its boundary
 * at t = fp32(t0 + n * dt_i), dt_i the grid's float time step widened to double,
 * as a per-grid loop calling the boundary with that time; each grid's result is
 * bit-identical to pde_heat_rollout_at with those times.  pde_batch_rollout
 * refuses such plans (PDE_ERR_UNSUPPORTED). */
int pde_batch_rollout_at(const PdeBatchPlan* plan, int32_t nsteps, double t0, void* stream);

/* ---- immersed boundary (FDM/boundary/immersedBoundary.py) ----
 * Solid regions inside the grid given by an int8 bitmask (X, Y, Z), nonzero =
 * solid, with the reference's staircase boundary.  Solid cells must not lie on
 * the array's outer layer along an eligible axis (the reference reads outside
 * the array there): such bitmasks give PDE_ERR_ARG. */

/* Scratch bytes pde_ib_maps needs for a grid (-1 for an invalid grid). */
int64_t pde_ib_work_bytes(const PdeGrid* grid);

/* The index maps of finalize() (immersedBoundary.py:57-151, kernels :344-438),
 * each list in C order as the reference's np.nonzero / np.unique give them:
 *   solid_boundary  (n_sb x 3 int32): solid cells with a fluid neighbour along an eligible axis
 *   fluid_neighbors (n_sb x D x 2 int8): the bitmask at -1 / +1 along each eligible axis
 *   interior_solids (n_is x 3 int32): the other solid cells
 *   fluid_boundary  (n_fb x 3 int32): fluid cells next to a solid cell
 * counts[3] receives (n_sb, n_is, n_fb).  With solid_boundary NULL only the counts
 * are computed (size the lists, then call again).  Synchronises the stream (the
 * counts come back to the host); not for stream capture.  work: pde_ib_work_bytes. */
int pde_ib_maps(const int8_t* bitmask, const PdeGrid* grid, int32_t* solid_boundary,
                int8_t* fluid_neighbors, int32_t* interior_solids, int32_t* fluid_boundary,
                int64_t* counts, void* work, int64_t work_bytes, void* stream);

/* forward(u, fill_value) of the immersed boundary (immersedBoundary.py:176-298):
 * out = in (copied unless out == in), then for each boundary cell and component
 * (bc_type / bc_value: n_boundary x ncomp, row-major) PDE_BC_DIRICHLET sets the
 * value and PDE_BC_VON_NEUMANN the running mean over the fluid neighbours of
 * (u_f - (s * value) * dx), s = -1 / +1, every operation rounded on its own (other
 * types leave the cell as it is); then every interior solid cell takes fill_value
 * in all components.  out may equal in.  Bit-identical to the reference. */
int pde_ib_apply(const float* in, float* out, const PdeGrid* grid, int32_t ncomp,
                 const int32_t* solid_boundary, const int8_t* fluid_neighbors,
                 const int8_t* bc_type, const float* bc_value, int64_t n_boundary,
                 const int32_t* interior_solids, int64_t n_interior, float fill_value,
                 void* stream);

/* ---- element-wise and absorbing-layer operators (weakly compressible / ACM path) ---- */

/* OuterProduct (FDM/module/elementWiseOps.py:10-48): per cell c,
 * out[c][i][j] = a[c][i] * b[c][j]; a: cells x na, b: cells x nb, out: cells x na x nb. */
int pde_outer(const float* a, const float* b, float* out, int64_t cells, int32_t na, int32_t nb,
              void* stream);

/* scalarVectorMult (elementWiseOps.py:51-88, FDM/kernel/elementWiseOps.py:6-23):
 * out[c][k] = s[c] * b[c][k]; s: one float per cell, b and out: cells x nb. */
int pde_scalar_mult(const float* s, const float* b, float* out, int64_t cells, int32_t nb, void* stream);

/* FarField / ViscousDampingLayer on their layer points (FDM/kernel/farfield.py:50-77,
 * FDM/kernel/viscousDampingLayer.py:50-76).  For point p (flat cell index cells[p],
 * ncomp floats per cell) and component k, with damp = scale * profile[p]:
 *   cond_host != NULL (FarField):    out = -damp * (in - cond_host[k])
 *   cond_host == NULL (damping):     out = -damp * in
 * each operation rounded on its own; other cells of out are not written.
 * profile[p] = (dx / L) ** exponent, the layer depth of the point over its
 * thickness, prepared by the caller (once per layer).  cond_host: up to 16 host
 * floats (the far-field vector or matrix), copied into the launch. */
int pde_layer_apply(const float* in, float* out, int32_t ncomp, const int64_t* cells,
                    const float* profile, int64_t npoints, float scale, const float* cond_host,
                    void* stream);

/* Allocation-free variant of pde_heat_rollout.  No counterpart in the
 * reference.  For callers that cannot allocate device memory (a memory manager
 * owns every allocation, cudaMalloc is not allowed in a latency-critical loop,
 * or a foreign-language host can only pass the field buffers it holds): the
 * scratch field comes from a fixed device array inside this library, of
 * PDE_NOALLOC_MAX_FLOATS floats (16 MiB), held on every GPU that loads the
 * library until the process exits.  Grids with X*Y*Z*ncomp above that return
 * PDE_ERR_TOO_LARGE.  The first call in a CUDA context looks the array up
 * (cudaGetSymbolAddress) and should come before any stream capture; the
 * address is kept per context (by its unique id), so a new context, or the
 * primary context again after cudaDeviceReset, looks it up anew.  All calls
 * share the array: calls that overlap on the GPU race, so serialise them.
 * Arguments and results are those of pde_heat_rollout without `work`. */
#define PDE_NOALLOC_MAX_FLOATS (1 << 22)
int pde_heat_rollout_noalloc(const float* u_in, float* u_out, const PdeGrid* grid, int32_t ncomp,
                             const PdeBCRules* rules, float alpha, float dt, int32_t nsteps,
                             int32_t steps_per_pass, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PDE_B200_H */
