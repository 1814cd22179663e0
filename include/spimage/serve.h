/*
 * Reconstruction server (no counterpart in the reference, which runs one
 * SpPhaser at a time on the legacy default stream; its Python Reconstructor
 * loops over random starts sequentially, src/_spimage_reconstructor.py:677-740).
 *
 * A server owns one host worker thread.  Jobs are submitted from any thread;
 * each job is one pattern with `starts` independent random starts and an
 * algorithm schedule.  The worker admits pending jobs while the number of jobs
 * on the GPU is below max_active_jobs and the device memory the jobs hold
 * stays within hbm_budget_bytes (first fit in arrival order), keeps every
 * admitted job's iterates, support and mask resident in its own device
 * context on its own CUDA stream, and advances the jobs chunk by chunk, so the
 * work of different jobs overlaps on the device.  Contexts of finished jobs
 * are kept and reused by later jobs of the same shape; idle contexts of other
 * shapes are freed when a job would not fit otherwise.
 *
 * A job runs through the SpPhaser API (sp_phaser_set_starts,
 * sp_phaser_init_models_device, sp_phaser_iterate), so its results are bit for
 * bit those of the same schedule run alone.
 *
 * Failure handling: a job ends early, with a negative status and an error
 * text, when its work fails on the device (SPB_JOB_FAILED; its context is
 * freed), when it is cancelled (SPB_JOB_CANCELLED), when a model of one of
 * its starts holds NaN or infinite values after a chunk (SPB_JOB_NONFINITE:
 * every chunk is followed by a check on the job's stream), or when its
 * wall-clock budget since submission runs out (SPB_JOB_EXPIRED).  Running
 * jobs stop at their next chunk boundary, after the chunks already on the
 * GPU; the server and the other jobs carry on.  The reference's phaser
 * returns negative codes for its own errors (src/phasing.c:898-998) and
 * exits on CUDA errors; here no job's failure ends the process.
 *
 * Return values: 0 success, negative error; the error text of a call is
 * spb_server_last_error(), that of a failed job spb_server_job_error().
 */
#ifndef SPB_SERVE_H
#define SPB_SERVE_H 1
#ifdef __cplusplus
extern "C" {
#endif

typedef struct spb_server spb_server;

typedef struct {
  double hbm_budget_bytes; /* device memory for job contexts; 0: 60% of the free memory at creation */
  int max_active_jobs;     /* jobs on the GPU at once; 0: 8 */
  int chunk_slots;         /* iteration slots per enqueued chunk; 0: 100 */
  int chunks_ahead;        /* chunks queued per job ahead of the GPU; 0: 2 */
  int no_autotune;         /* 1: keep the built-in launch shapes; 0: tune them (sp_phaser_autotune) for the
                              first stage's algorithm of every new (shape, starts, algorithm) */
} spb_server_config;

enum { SPB_JOB_MAX_STAGES = 4 };

typedef struct {
  int algorithm;  /* SpHIO, SpRAAR, SpDiffMap (Elser's gammas) or SpER */
  float beta;     /* constant beta of HIO, RAAR and the difference map */
  int iterations; /* iteration slots of this stage (support updates use slots) */
} spb_job_stage;

typedef struct {
  int nx, ny, nz;
  int starts;             /* independent random starts */
  const float *amplitudes; /* [N] measured amplitudes, reciprocal space shifted */
  const int *mask;         /* [N] nonzero where the amplitude is measured */
  const int *support;      /* [N] nonzero inside the initial support */
  int constraints;         /* SpPhasingConstraints */
  int nstages;
  spb_job_stage stage[SPB_JOB_MAX_STAGES];
  int support_period;     /* area support update every this many slots; 0: none */
  float support_area;     /* area fraction of the support update */
  float blur_start, blur_end; /* blur radius, Bezier from the first to the last slot */
  unsigned long long seed; /* start b gets random phases keyed by seed + b (device Philox4x32-10) */
  int keep_models;        /* 1: keep every start's final model for spb_server_result */
  double time_budget_s;   /* wall-clock seconds from submission after which the job ends as
                             SPB_JOB_EXPIRED; 0: no limit */
} spb_job;

/* spb_job_info.status */
enum {
  SPB_JOB_DONE = 0,
  SPB_JOB_RUNNING = 1,     /* pending or running */
  SPB_JOB_FAILED = -1,     /* device or set-up error */
  SPB_JOB_CANCELLED = -2,  /* spb_server_cancel */
  SPB_JOB_NONFINITE = -3,  /* NaN or infinity in a model */
  SPB_JOB_EXPIRED = -4     /* time_budget_s ran out */
};

typedef struct {
  int status;    /* SPB_JOB_DONE, SPB_JOB_RUNNING or a negative SPB_JOB_* code */
  int starts;
  long long slots; /* iteration slots per start */
  double t_submit, t_admit, t_finish; /* seconds since the server was created; -1 if not reached */
} spb_job_info;

int spb_server_create(spb_server **srv, const spb_server_config *cfg);
/* finishes every submitted job, then frees the server */
void spb_server_destroy(spb_server *srv);
/* copies the job's inputs; returns the job id (>= 0) or -1 */
long long spb_server_submit(spb_server *srv, const spb_job *job);
/* waits until the job has finished or timeout_s has passed (timeout_s < 0:
 * no limit); info->status tells which; returns -1 for an unknown id */
int spb_server_wait(spb_server *srv, long long id, double timeout_s, spb_job_info *info);
/* Cancels a job: a pending job ends at once, a running one at its next
 * chunk boundary (its context stays reusable).  Returns -1 for an unknown id
 * or a job that has already ended. */
int spb_server_cancel(spb_server *srv, long long id);
/* results of a finished job: final Fourier error and support fraction of
 * every start ([starts] each) and, if the job kept them, the models
 * ([starts][N] complex, interleaved re/im); NULL skips an output.  Releases
 * a finished or failed job (a failed one returns -1 with its error): its id
 * is unknown afterwards. */
int spb_server_result(spb_server *srv, long long id, float *efourier, float *support_fraction, float *models);
/* counters: [0] jobs finished, [1] start-slots finished (starts x slots),
 * [2] most jobs on the GPU at once, [3] most bytes of contexts held,
 * [4] contexts created, [5] contexts freed to make room, [6] contexts reused,
 * [7] jobs failed */
int spb_server_stats(spb_server *srv, double stats[8]);
const char *spb_server_last_error(void);
const char *spb_server_job_error(spb_server *srv, long long id);

/* Device bytes a context of nb starts of nx*ny*nz holds (dm: with the
 * difference map's second transform pair). */
long long spb_ctx_footprint(int nx, int ny, int nz, int nb, int dm);

#ifdef __cplusplus
}
#endif
#endif
