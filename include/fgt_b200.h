/*
 * fgt_b200.h -- C ABI of the B200 (sm_100a) discrete point fast Gauss
 * transform.  Plain pointers and sizes only; no C++ or torch types.
 *
 * The drop-in entry point replaces the reference Fortran subroutine
 *   subroutine pfgt(nd,dim,delta,eps,iperiod,bs0,cen0,ns,sources,
 *                   ifcharge,charge,ifdipole,rnormal,dipstr,ifpgh,pot,grad,
 *                   hess,nt,targ,ifpghtarg,pottarg,gradtarg,hesstarg)
 * of src/pfgt/pfgt.f:6-10 (argument meaning: src/pfgt/pfgt.f:11-53).
 *
 * Array layouts are those of the reference (Fortran column-major, 4-byte
 * integers): sources(dim,ns) -> sources[i*dim+k], charge(nd,ns) ->
 * charge[i*nd+id], grad(nd,dim,n) -> grad[(i*dim+k)*nd+id],
 * hess(nd,nhess,n) -> hess[(i*nhess+m)*nd+id], nhess = dim*(dim+1)/2, hessian
 * order xx,yy,zz,xy,xz,yz (3D) and xx,xy,yy (2D) (src/pfgt/pfgt.f:52-53).
 * Outputs are overwritten for the requested fields only; unrequested output
 * arrays are never touched (length-1 dummies are fine), as in
 * src/pfgt/pfgt.f:378-406.  bs0/cen0 are outputs in free space (iperiod=0)
 * and inputs when periodic (src/common/pts_tree_nd.f:1350-1360).
 */
#ifndef FGT_B200_H
#define FGT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FGT_OK 0
#define FGT_ERR_ARG 1         /* invalid argument */
#define FGT_ERR_CUDA 2        /* CUDA runtime error */
#define FGT_ERR_NOMEM 3       /* device or host allocation failed */
#define FGT_ERR_UNSUPPORTED 4 /* valid input outside the supported range */
#define FGT_ERR_TIMEOUT 5     /* a bounded device wait gave up */
#define FGT_ERR_NODEVICE 6    /* no CUDA device / library not usable */
#define FGT_ERR_INJECTED 7    /* host-side fault injection (FGT_FAULT) */
#define FGT_ERR_CHECK 8       /* a device bounds check failed (FGT_CHECK build only) */

/* precision policy */
#define FGT_PREC_AUTO 0  /* mixed FP32 bulk when eps >= 1e-6, FP64 otherwise */
#define FGT_PREC_FP64 1  /* whole pipeline in FP64 */
#define FGT_PREC_MIXED 2 /* FP32 bulk with FP64 geometry and accumulation */

/* per-call statistics (filled when fgt_opts.stats != NULL) */
typedef struct fgt_stats {
  int nlevels, nboxes, npwlevel, npw, ndiv;
  int precision_used;    /* FGT_PREC_FP64 or FGT_PREC_MIXED */
  int n_form_boxes;      /* boxes that form a plane-wave expansion */
  int n_eval_boxes;      /* boxes with a local plane-wave expansion */
  int n_eval_nufft;      /* ... evaluated through the interpolation grid */
  int n_translations;    /* sum over boxes of the PW list length */
  int spread_width;      /* kernel width of the spreader */
  int grid_cells;        /* spreading sub-grid cells per dimension */
  int n_kernel_launches; /* kernels launched by this call */
  double near_pairs;     /* source/target pairs of the direct near field */
  /* algorithmic work of the call (FP32 or FP64 flops, HBM bytes) */
  double flops_form;     /* spreading stencils + DFT passes of the form kernel */
  double flops_eval;     /* DFT passes + interpolation stencils + modal sums */
  double flops_direct;   /* near-field pair arithmetic */
  double bytes_translate;/* expansion traffic of the translation kernel */
  double pts_form, pts_eval_nufft, pts_eval_modal;
  double bs0, cen0[3];
  /* milliseconds on the device stream: 0 h2d, 1 tree, 2 sort+gather,
   * 3 lists, 4 form, 5 translate, 6 eval, 7 direct, 8 scatter, 9 d2h,
   * 10 total */
  double ms[12];
  int small_eval_used;   /* modal-evaluation threshold the call used */
  int tuned;             /* 1: parameters came from the tuning cache or a tuning run */
  int slabs_form;        /* x-slabs per form sub-grid (1: whole grids) */
  int slabs_eval;        /* x-slabs per evaluation sub-grid (1: whole grids) */
} fgt_stats;

typedef struct fgt_opts {
  int precision;    /* FGT_PREC_* */
  int device_ptrs;  /* 1: every array argument is a device pointer on `device` */
  int device;       /* CUDA device ordinal, -1 = current device */
  void *stream;     /* cudaStream_t to run on; NULL = the library's stream */
  int ndiv;         /* max sources per unrefined box; 0 = reference value
                       20/80/250 for dim 1/2/3 (src/pfgt/pfgt.f:122-128) */
  int small_eval;   /* boxes with at most this many evaluation points use
                       direct modal evaluation; -1 = tuned default */
  int spread_width; /* spreading kernel width in grid cells; 0 = from eps */
  int timing;       /* 1: record per-phase times into stats->ms */
  fgt_stats *stats; /* optional output */
  int root_level;   /* free space only: >= 0 makes bs0/cen0 inputs and this
                       the cut-off level (the root box pts_tree_boxsize0,
                       src/common/pts_tree_nd.f:1330-1414, computed on a
                       larger point set this call is a spatial shard of);
                       -1 (default) = computed from the points */
  int autotune;     /* 0 off (default); 1 take tuned parameters from the
                       cache; 2 also tune on a cache miss: the call times the
                       strength-dependent part with each candidate (small_eval
                       thresholds; worker counts in fgt_pfgt_batch), keeps the
                       fastest in the cache and returns its results.  Cache:
                       the file named by FGT_TUNE_CACHE, else
                       $HOME/.cache/fgt_b200/tune.txt.  Applies only to
                       parameters left at their defaults. */
} fgt_opts;

/* Fill *opts with defaults (precision AUTO, host pointers, current device). */
void fgt_opts_default(fgt_opts *opts);

/*
 * Point FGT with status return.  Same arguments and semantics as the
 * reference pfgt (src/pfgt/pfgt.f:6-409) passed by value/pointer, plus the
 * options pointer (NULL = defaults).  Returns FGT_OK or an FGT_ERR_* code.
 */
int fgt_pfgt_c(const fgt_opts *opts, int nd, int dim, double delta, double eps,
               int iperiod, double *bs0, double *cen0, int ns,
               const double *sources, int ifcharge, const double *charge,
               int ifdipole, const double *rnormal, const double *dipstr,
               int ifpgh, double *pot, double *grad, double *hess, int nt,
               const double *targ, int ifpghtarg, double *pottarg,
               double *gradtarg, double *hesstarg);

/*
 * One instance of a batched call: the arguments of the reference pfgt
 * (src/pfgt/pfgt.f:6-10) by value/pointer, plus its status on return.
 */
typedef struct fgt_instance {
  int nd, dim;
  double delta, eps;
  int iperiod;
  double *bs0, *cen0;
  int ns;
  const double *sources;
  int ifcharge;
  const double *charge;
  int ifdipole;
  const double *rnormal, *dipstr;
  int ifpgh;
  double *pot, *grad, *hess;
  int nt;
  const double *targ;
  int ifpghtarg;
  double *pottarg, *gradtarg, *hesstarg;
  int status; /* out: FGT_OK or FGT_ERR_* of this instance */
} fgt_instance;

/*
 * Many independent point FGTs (the batched workload of the reference's test
 * scenarios: a loop of pfgt calls, src/pfgt/pfgt.f:6-409 each) in one call.
 * Every instance gives the results of fgt_pfgt_c with the same options; the
 * options' stream, stats and timing fields are ignored.  Instances run
 * concurrently on `nworkers` host worker threads, each with its own stream
 * and device workspace (<= 0: 12, at most the host's threads), largest
 * instances first.  Returns when all instances are done: FGT_OK, or the
 * first failing instance's status (each instance's own status is in its
 * `status` field).
 */
int fgt_pfgt_batch(const fgt_opts *opts, int ninst, fgt_instance *inst, int nworkers);

/*
 * Reusable plan: the point-dependent part of pfgt kept on the device for
 * repeated calls on the same sources and targets with new strengths.  The
 * reference repeats all of it on every call: scalar set-up and tree
 * (src/pfgt/pfgt.f:110-321, src/common/pts_tree_nd.f:35-1256), lists
 * (src/common/tree_routs_nd.f:1063-1555) and the sort of the points
 * (src/common/fmmcommon2d.f:3-27).
 *
 * fgt_plan_create takes the geometry arguments of pfgt (bs0/cen0 written in
 * free space, read when periodic) and the options (precision, device
 * pointers, device, stream, ndiv, small_eval, spread_width are kept; stats
 * and timing are ignored); *status receives FGT_OK or an FGT_ERR_* code and
 * NULL is returned on failure.  fgt_plan_execute takes the strength and
 * output arguments of pfgt (same layouts; host or device pointers as at
 * creation) and gives the results of fgt_pfgt_c on the plan's points.  One
 * plan may be executed from several host threads at once (each thread runs
 * on its own stream and workspace unless the plan was given a stream).
 * fgt_plan_destroy releases the plan's device memory.
 */
typedef struct fgt_plan fgt_plan;
fgt_plan *fgt_plan_create(const fgt_opts *opts, int nd, int dim, double delta,
                          double eps, int iperiod, double *bs0, double *cen0,
                          int ns, const double *sources, int nt,
                          const double *targ, int *status);
int fgt_plan_execute(fgt_plan *plan, int ifcharge, const double *charge,
                     int ifdipole, const double *rnormal, const double *dipstr,
                     int ifpgh, double *pot, double *grad, double *hess,
                     int ifpghtarg, double *pottarg, double *gradtarg,
                     double *hesstarg);
void fgt_plan_destroy(fgt_plan *plan);

/*
 * gfortran-mangled drop-in for `call pfgt(...)` (src/pfgt/pfgt.f:6-10): all
 * 24 arguments by reference, no hidden string lengths.  The reference has no
 * error argument; on failure the requested outputs are NaN-filled and the
 * status is kept for fgt_last_status().
 */
void pfgt_(const int *nd, const int *dim, const double *delta,
           const double *eps, const int *iperiod, double *bs0, double *cen0,
           const int *ns, const double *sources, const int *ifcharge,
           const double *charge, const int *ifdipole, const double *rnormal,
           const double *dipstr, const int *ifpgh, double *pot, double *grad,
           double *hess, const int *nt, const double *targ,
           const int *ifpghtarg, double *pottarg, double *gradtarg,
           double *hesstarg);

/*
 * gfortran-mangled drop-in for `call pfgt_direct(...)` (src/pfgt/pfgt.f:
 * 1156-1159): adds the direct Gaussian interactions of sources
 * istart..iend onto targets jstart..jend (1-based, inclusive), cut off at
 * squared distance dmax; periodic (iperiod=1) shifts the sources by
 * shifts(dim).  Computed on the GPU in FP64.  Outputs are incremented.
 */
void pfgt_direct_(const int *nd, const int *dim, const double *delta,
                  const double *dmax, const int *iperiod, const double *shifts,
                  const int *istart, const int *iend, const int *jstart,
                  const int *jend, const double *source, const int *ifcharge,
                  const double *charge, const int *ifdipole,
                  const double *rnormal, const double *dipstr,
                  const double *targ, const int *ifpgh, double *pot,
                  double *grad, double *hess);

/*
 * Allocation-free variant of the FP64 all-pairs direct sum behind
 * pfgt_direct_; it has no counterpart in the reference.  For callers that
 * cannot allocate device memory: it calls no cudaMalloc, cudaFree or other
 * allocating routine.  All arrays are DEVICE pointers owned by the caller,
 * in pfgt_direct's layouts (sources(dim,ns), charge(nd,ns), rnormal(dim,ns),
 * dipstr(nd,ns), targ(dim,nt), pot(nd,nt), grad(nd,dim,nt),
 * hess(nd,nhess,nt)); the outputs are incremented.  shifts: host array of
 * dim doubles added to the sources (periodic images), or NULL.  Sources
 * closer than sqrt(dmax) interact.  Runs asynchronously on `stream` (a
 * cudaStream_t; NULL = the legacy default stream) and returns FGT_OK or an
 * FGT_ERR_* code (message in fgt_last_error()).
 *
 * Scratch is a static device array of FGT_NOMALLOC_SCRATCH_BYTES that every
 * GPU loading the library holds until exit: nt*nd*(1 + dim*[ifpgh>=2] +
 * nhess*[ifpgh>=3]) doubles must fit in it, else FGT_ERR_UNSUPPORTED.  The
 * first call on each device loads the library's module there (CUDA loads
 * modules lazily, so that is when the GPU reserves the array) and resolves
 * the array's address with cudaGetSymbolAddress.  Make that first call
 * before the host gives the GPU's memory to its own pool and before any
 * stream capture; a call with nt = 0 or ns = 0 does exactly this and
 * computes nothing.
 * All calls share the array (it is cleared at the start of each call):
 * calls that overlap on the GPU, on any streams, race.
 */
#define FGT_NOMALLOC_SCRATCH_BYTES (8u << 20)
int fgt_direct_nomalloc(int nd, int dim, double delta, double dmax,
                        const double *shifts, int ns, const double *sources,
                        int ifcharge, const double *charge, int ifdipole,
                        const double *rnormal, const double *dipstr, int nt,
                        const double *targ, int ifpgh, double *pot,
                        double *grad, double *hess, void *stream);

/* Status of the last pfgt_/pfgt_direct_ call on this host thread. */
int fgt_last_status(void);

/* Human-readable message of the last error on this host thread. */
const char *fgt_last_error(void);

/* Library version string. */
const char *fgt_version(void);

/*
 * Introspection of the device-built tree and interaction lists (test and
 * debugging support).  Builds the tree and lists of a pfgt call with the
 * given arguments (host pointers) and keeps a host copy.  Returns NULL when
 * no device is usable.  The tree replaces pts_tree_mem/pts_tree_build/
 * pts_tree_sort (src/common/pts_tree_nd.f:35-644, 1226-1256); the lists
 * replace pfgt_find_pwexp_boxes, pfgt_compute_listpw and
 * pfgt_compute_modified_list1 (src/common/tree_routs_nd.f:1063-1555).
 * Box ids are 0-based in level-major order, keys ascending within a level.
 */
void *fgt_debug_tree_build(int dim, double delta, double eps, int iperiod,
                           double bs0, const double *cen0, int ns,
                           const double *sources, int nt, const double *targ,
                           int ndiv);
/* Copies array `name` (see fgt_b200/__init__.py for the list) into dst
 * (at most cap elements) and returns its length; dst may be NULL. */
long fgt_debug_tree_get(void *h, const char *name, void *dst, long cap);
void fgt_debug_tree_free(void *h);

/*
 * Self-test of the device bounds checks (test support; no counterpart in the
 * reference, which has no checks).  libfgt_b200_check.so, the FGT_CHECK
 * build, checks the indexed accesses of its kernels on the device: a failed
 * check records a site number and skips the access (no trap), and the call
 * returns FGT_ERR_CHECK naming the first site.  This entry point runs one
 * kernel on a host-crafted out-of-range index and returns FGT_ERR_CHECK in
 * that build, FGT_ERR_UNSUPPORTED in the normal one.
 */
int fgt_check_selftest(void);

#ifdef __cplusplus
}
#endif

#endif /* FGT_B200_H */
