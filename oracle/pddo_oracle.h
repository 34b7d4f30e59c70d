/* Test infrastructure only (the oracle).  A plain-C CPU restatement of PeriX's PDDO hot path, used by
 * tests/, the smoke check and bench.py's CPU-baseline leg to check results.  The product never links it.
 * Node ids are 1-based in family lists (reference convention); everything else is 0-based.
 * Each function cites the reference file:line whose algorithm it restates. */
#ifndef PDDO_ORACLE_H
#define PDDO_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* multi-index list (PDOperators.cpp:51-75): returns nop; pqr[3*k..] = (p,q,r), fact[k] = p!q!r! */
int orc_qindices(int dim, int order, int *pqr, int *fact);

/* families (CreatePDMesh.cpp:910-1082), uniform horizon.  Two-pass: call with ids==NULL to get counts in
 * off[0..n] (off[0]=0, prefix sums), then again with ids sized off[n].  cut(i1,j1) crack hook: the
 * crack test of PDMesh.cpp:104-159 over segments/planes and the ghost mirror map `mirror` (0 for bulk);
 * no cracks disables it.  Returns number of directed bonds. */
long long orc_families(int n, const double *coords3, double radius, int is3d, int ncracks, const double *cracks,
                       int nplanes, const double *planes, const int *mirror, int force_only, int *off, int *ids);

/* PDMesh.cpp:104-159: xy segments (4 doubles each) and bounded quads (12 doubles each) */
int orc_crack_cuts(int n, const double *coords3, const int *mirror, int ncracks, const double *cracks, int nplanes,
                   const double *planes, int i1, int j1);

/* g-functions (CalcPDOperators.cpp:108-226 + 307-354): ops[bond*nop+k].  degenerate[i] set as the
 * reference's m_LastFamilyDegenerate (usable bonds < nop, or solve inconsistency > 1e-8 relative).
 * deep ghost zeroing is not applied (single ghost layer).  Returns number of degenerate nodes. */
int orc_gbuild(int n, int dim, int order, const double *coords3, const double *vols, const int *off,
               const int *ids, double delta, double dx_char, int volume_correction, double *ops,
               unsigned char *degenerate);

/* D^k u_i = sum_t g^k_it (u_j - u_i) over all nop slots (PoissonElement.cpp:67-105 pattern) */
void orc_apply(int n, int nop, const int *off, const int *ids, const double *ops, const double *u, double *out);

/* CSR pattern (SparseMatrix.cpp:73-185): rowptr sized n*ndof+1; cols==NULL => only rowptr. Returns nnz. */
long long orc_csr_pattern(int n, int ndof, const int *off, const int *ids, const int *mirror, int *rowptr,
                          int *cols);

/* Poisson CSR values, K=-dF/dU, RHS=+F (FormResidualAndJacobianParallel.cpp:114-171 +
 * PoissonElement.cpp:26-58), per-node source f.  slot lookup by binary search (SparseMatrix.cpp:187-196). */
void orc_poisson_assemble(int n, int dim, int nop, const int *lapslots /*2 or 3 slot ids*/, const int *off,
                          const int *ids, const double *ops, double sigma, const double *f, const double *u,
                          const int *rowptr, const int *cols, double *kvals, double *rhs);

/* explicit_pddo_frac rate (ExplicitPDDOFracElement.cpp:239-299): damage at u then Navier force.
 * navier[bond*c+..] = 2D {Gxx,Gyy,Gxy}, 3D {Gxx,Gyy,Gzz,Gxy,Gxz,Gyz}; health in/out (1.0/0.0). */
void orc_epf_rate(int n, int dim, const double *coords3, const int *off, const int *ids, const double *navier,
                  double C11, double C12, double C66, double rho, const double *b, double sc, int tension_only,
                  int damage_on, const double *u, double *health, double *accel);

/* elastic constants (ExplicitPDDOFracElement.cpp:38-53) -> C[3]; critical stretch from G0
 * (FractureCriterion.h:30-43) */
void orc_elastic_constants(int dim, int plane_stress, double E, double nu, double *C);
double orc_critical_stretch(int dim, int plane_stress, double G0, double E, double delta);

/* ghost BC preset program (DirichletBC.cpp:107-147, NeumannBC.cpp:88-105, BCSystem.cpp:114-129);
 * same encoding as ref_bc_preset in ref_harness.cpp. */
void orc_bc_preset(int n, int dim, const double *coords3, const int *mirror, int nbc, const int *kind,
                   const int *comp_mask, const int *direct, const double *val, const double *vel,
                   const int *has_box, const double *box, const int *node_off, const int *nodes, double t,
                   double *u);

/* central difference (TimeStepping.cpp:479-547), nsteps uniform steps, BC after each step */
void orc_epf_run(int n, int dim, const double *coords3, const int *mirror, const int *off, const int *ids,
                 const double *navier, double C11, double C12, double C66, double rho, const double *b,
                 double sc, int tension_only, int damage_on, const double *u0, const double *v0, double dt,
                 int nsteps, int nbc, const int *kind, const int *comp_mask, const int *direct, const double *val,
                 const double *vel, const int *has_box, const double *box, const int *node_off, const int *nodes,
                 double *u, double *uold, double *health);

#ifdef __cplusplus
}
#endif
#endif
