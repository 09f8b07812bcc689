/*
 * casim_b200 — C ABI of the B200-native CaSim release-site hot path.
 *
 * One handle owns a batch of independent release sites (dyads) resident on one
 * GPU: the cleft reaction-diffusion fields, RyR gating states and their
 * MRG32k3a streams, the jSR pool and the cytosol (well-mixed pool or 3D grid).
 * A call to casim_b200_step() advances every site by n explicit time steps
 * entirely on the device; nothing crosses PCIe inside the time loop.
 *
 * Plain C types only. Every call returns a casim_status; on failure
 * casim_b200_last_error() describes it. Handles are not thread-safe: one host
 * thread drives one handle (the reference drives its GPU classes from one
 * thread too, CaSim/ParallelHybridSolver.cpp:373-405).
 *
 * Node order used by every field getter/setter is the reference's:
 *   2D: y + ny*x            (CaSim/DyadRD2DCPU.cpp:270-272)
 *   3D: z + nz*(y + ny*x)   (CaSim/DyadRDCPU.cpp:277-279)
 * Species order: ions (JSON key order), then ion-buffer pairs (ion-major,
 * buffer-minor, CaSim/DyadRD2DCPU.cpp:83-99), then free buffers.
 */
#ifndef CASIM_B200_H
#define CASIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct casim_b200_sim* casim_h;

typedef enum {
    CASIM_OK = 0,
    CASIM_EINVAL = 1,      /* malformed JSON, bad argument, out-of-range site/channel */
    CASIM_ECUDA = 2,       /* a CUDA runtime call failed (message carries cudaGetErrorString) */
    CASIM_ENOMEM = 3,      /* device allocation failed */
    CASIM_EUNSTABLE = 4,   /* explicit scheme violates dt*sum(2D/h^2) <= 1 for some species */
    CASIM_ETIMEOUT = 5,    /* a bounded device wait gave up */
    CASIM_ENONFINITE = 6,  /* a NaN/Inf was found in the state by casim_b200_check_finite */
    CASIM_EUNSUPPORTED = 7 /* configuration outside this build's limits */
} casim_status;

typedef enum { CASIM_FP64 = 0, CASIM_FP32 = 1 } casim_precision;

/* Which device path steps the batch.
 * PLAIN:    one time step per launch sequence (cytosol/jSR/gating, RD stencil,
 *           coupling), fields in HBM. Any site size.
 * RESIDENT: each site lives in one thread block's shared memory for the whole
 *           call; all time steps run inside one persistent launch.
 * AUTO:     PLAIN for 3D clefts or a 3D cytosol whose state (one copy of the
 *           fields and the cytosol) is larger than the device's L2 cache and whose
 *           species layout the streaming kernels serve (1-2 ions, at most 4 pairs,
 *           1 or 3 cleft layers at every site): there the resident kernel's per-step
 *           chain of phases is slower than streaming the state from HBM. Otherwise
 *           RESIDENT when every site fits, else PLAIN. casim_b200_path_note says
 *           which rule chose. */
typedef enum { CASIM_PATH_AUTO = 0, CASIM_PATH_PLAIN = 1, CASIM_PATH_RESIDENT = 2 } casim_path;

/* Optional per-site table (struct of arrays). Any NULL member falls back to
 * the JSON: grid extents from x/dx+1, y/dy+1, z/dz+1 (CaSim/DyadRD2DCPU.cpp:17-18),
 * RyR coordinates from the "Coordinates" file, seeds from "Seed", jSR from
 * "jSR"/"Ions"/<ion>/"Concentration". */
typedef struct casim_site_table {
    int32_t n_sites;
    const int32_t* nx;         /* grid nodes along x per site */
    const int32_t* ny;
    const int32_t* nz;         /* 3D only */
    const int32_t* n_channels; /* RyRs per site */
    const double* ch_x;        /* RyR coordinates in nm, concatenated site after site */
    const double* ch_y;
    const uint32_t* seeds;     /* 6 MRG32k3a seed words per site */
    const double* jsr_init;    /* n_ions values per site */
} casim_site_table;

typedef struct casim_info {
    int32_t n_sites;
    int32_t dim;               /* 2 or 3 */
    int32_t n_ions;
    int32_t n_pairs;
    int32_t n_buffers;
    int32_t n_cyto_species;    /* cytosol pool: n_ions + cytosol pairs; RD3D: same, per node */
    int32_t cyto_nodes;        /* RD3D nodes per site (mc^3), 0 for the pool */
    int32_t precision;
    int32_t path;              /* the path actually used */
    int32_t max_channels;
    int64_t total_nodes;       /* cleft nodes over all sites */
    double dt_ms;
    double element_volume;     /* nm^3, as DyadSeries::GetElementVolume */
} casim_info;

/* Build a batch from a reference-schema Parameters.json text.
 * Replaces the compartment construction in ParallelHybridSolver's constructor
 * (CaSim/ParallelHybridSolver.cpp:13-131) for the dyad, jSR, nSR and cytosol.
 * base_dir resolves relative "Coordinates" paths (may be NULL = cwd).
 * sites may be NULL: then "NumBatch" identical sites are built. */
casim_status casim_b200_create(const char* json_text, const char* base_dir, casim_precision precision,
                               casim_path path, const casim_site_table* sites, casim_h* out);
casim_status casim_b200_destroy(casim_h h);
casim_status casim_b200_info(casim_h h, casim_info* out);
/* Name of species `index` (ions, pairs as "<ion>-<buffer>", free buffers). */
casim_status casim_b200_species_name(casim_h h, int32_t index, char* buf, size_t n);
/* Name of cytosol species `index` (ions, then the cytosol's ion-buffer pairs as
 * "<ion>-<buffer>"), the keys of CytosolSeries::GetConcentrations
 * (CaSim/CytosolPool.cpp:331-357). */
casim_status casim_b200_cyto_species_name(casim_h h, int32_t index, char* buf, size_t n);
casim_status casim_b200_last_error(casim_h h, char* buf, size_t n);

/* Use this CUDA stream (a cudaStream_t) for all work of the handle; NULL = the
 * handle's own stream. */
casim_status casim_b200_set_stream(casim_h h, void* cuda_stream);

/* Reset every compartment to its initial state.
 * Replaces DyadSeries::Reset, SRSeries::Reset, CytosolSeries::Reset, NSRSeries::Reset
 * (CaSim/DyadSeries.h:19, CaSim/SRSeries.h:9, CaSim/CytosolSeries.h:15, CaSim/NSRSeries.h:8). */
casim_status casim_b200_reset(casim_h h);
/* DyadSeries::InitOpening(site, channel) (CaSim/DyadSeries.h:20, CaSim/DyadChannels.cpp:83-95):
 * consumes n_channels + 1 draws of the site's stream and opens `channel`. */
casim_status casim_b200_init_opening(casim_h h, int32_t site, int32_t channel);
/* The solver's Update() (CaSim/ParallelHybridSolver.cpp:159-175): mouth
 * gather, Dirichlet edges, efflux, RyR currents, pool coupling. */
casim_status casim_b200_update(casim_h h);
/* reset + init_opening(site, first_channel[site]) for every site + update, as
 * at the start of each batch in RunSimulations* (CaSim/ParallelHybridSolver.cpp:415-418). */
casim_status casim_b200_start(casim_h h, const int32_t* first_channel);
/* Per-site initial jSR concentrations (n_ions values per site) used by the
 * next reset/start: a new batch scenario without rebuilding the handle. */
casim_status casim_b200_set_site_jsr(casim_h h, const double* jsr_init);
/* Advance every site by n_steps time steps: per step the cytosol, dyad RD,
 * jSR, gating and Update of CaSim/ParallelHybridSolver.cpp:421-429.
 * Replaces DyadSeries::RunRD + RunMC + Update, SRSeries::Run/Update and
 * CytosolSeries::RunRD/Update for the whole batch. Asynchronous on the stream. */
casim_status casim_b200_step(casim_h h, int64_t n_steps);
casim_status casim_b200_synchronize(casim_h h);

/* ---- getters (synchronous; copy device state to host) ---- */
/* DyadSeries::GetConcentrations (CaSim/DyadSeries.h:29): one species of one
 * site, reference node order, nx*ny(*nz) doubles. */
casim_status casim_b200_get_field(casim_h h, int32_t site, int32_t species, double* out);
/* write one species of one site (reference node order); for tests and restarts */
casim_status casim_b200_set_field(casim_h h, int32_t site, int32_t species, const double* in);
/* DyadSeries::GetIonsNearChannels (CaSim/DyadSeries.h:31): mouth value of
 * `species` at every RyR of the site, as gathered by the last Update. */
casim_status casim_b200_get_mouth(casim_h h, int32_t site, int32_t species, double* out);
/* DyadSeries::GetChannelsStates (CaSim/DyadSeries.h:30): 0/1 per RyR. */
casim_status casim_b200_get_states(casim_h h, int32_t site, int32_t* out);
/* 60-state RyR models (SingleSiteMWC, CaSim/SingleSiteMWC.cpp): the micro-state
 * 0..59 of each RyR of the site (states 45-59 open); casim_b200_get_states gives
 * the open flags. EINVAL for two-state models. */
casim_status casim_b200_get_micro_states(casim_h h, int32_t site, int32_t* out);
/* Overwrites the open (1) / closed (0) state of every RyR of the batch
 * (site-major, as casim_b200_get_all_states returns them) without consuming
 * draws; call casim_b200_update afterwards so the currents follow. Generalises
 * DyadSeries::InitOpening (CaSim/DyadSeries.h:21), which opens one RyR per
 * site; used to hold arbitrary open sets (surrogate training snapshots). */
casim_status casim_b200_set_all_states(casim_h h, const int32_t* states);
/* SRSeries::GetIons (CaSim/SRSeries.h:12): jSR concentration per ion. */
casim_status casim_b200_get_jsr(casim_h h, int32_t site, double* out);
/* DyadSeries::GetTotalSRCurrent (CaSim/DyadSeries.h:24): per ion. */
casim_status casim_b200_get_total_current(casim_h h, int32_t site, double* out);
/* DyadSeries::GetEffluxes (CaSim/DyadSeries.h:23): n_ions + n_pairs values. */
casim_status casim_b200_get_efflux(casim_h h, int32_t site, double* out);
/* CytosolSeries::GetConcentrations (CaSim/CytosolSeries.h:19) for the pool:
 * n_ions + cytosol pairs values. */
casim_status casim_b200_get_cyto(casim_h h, int32_t site, double* out);
/* RD3D cytosol: one species of one site, mc^3 values, x fastest. */
casim_status casim_b200_get_cyto_field(casim_h h, int32_t site, int32_t species, double* out);
/* write one species of one site's RD3D cytosol (mc^3 values, x fastest); for
 * tests and restarts. No counterpart in the reference (it has no 3D cytosol). */
casim_status casim_b200_set_cyto_field(casim_h h, int32_t site, int32_t species, const double* in);
/* runif() draws consumed so far by the site's stream */
casim_status casim_b200_get_draws(casim_h h, int32_t site, uint64_t* out);
/* Ca released from the jSR so far (FP64 accumulator), in uM*nm^3 */
casim_status casim_b200_get_release(casim_h h, int32_t site, double* out);

/* Scan every site's cleft fields, RD3D cytosol grid and FP64 pool values (jSR,
 * cytosol pool, release accumulator) for NaN/Inf; returns CASIM_ENONFINITE and
 * the first bad site in *bad_site (or -1). No counterpart in the reference,
 * which checks nothing. */
casim_status casim_b200_check_finite(casim_h h, int32_t* bad_site);

/* Batched host views for drop-in output (CaSim/ParallelHybridSolver.cpp:316-337):
 * all sites' mouth Ca and channel states in one call each. */
casim_status casim_b200_get_all_mouth(casim_h h, int32_t species, double* out);  /* sum of channels */
casim_status casim_b200_get_all_states(casim_h h, int32_t* out);

/* Open-RyR traces recorded on the device. Replaces the host round trip of the
 * channel states at the output cadence (CaSim/ParallelHybridSolver.cpp:316-337)
 * that feeds the reference's release analysis. casim_b200_trace_enable allocates
 * [sites][max_samples] u16 counts, records sample 0 (the current states) and
 * then one sample every every_steps time steps of casim_b200_step (which stops
 * at each sample time; surrogate-gated windows are not sampled); sample j is at
 * j * every_steps * dt after the enable. Recording stops at max_samples. */
casim_status casim_b200_trace_enable(casim_h h, int64_t every_steps, int64_t max_samples);
casim_status casim_b200_trace_count(casim_h h, int64_t* n_samples);
/* out: [site][n_samples], n_samples from casim_b200_trace_count. */
casim_status casim_b200_get_open_traces(casim_h h, uint16_t* out);

/* Release-event analysis of the recorded traces on the device, with the
 * arithmetic of IndChannelCREAnalyzer::RunAnalysis
 * (CaSim/IndChannelCREAnalyzer.cpp:53-138), each site one trace:
 *   per_site [sites][5]: amplitude (most open RyRs), time to peak, time to end,
 *     integral of the open count (ms), its mean;
 *   histograms of open counts over time bins of hist_dt_ms (the reference's
 *     fixed 0.01 ms, CaSim/IndChannelCREAnalyzer.cpp:7), nh + 1 rows with
 *     nh = (long long)(max_time_ms / hist_dt_ms): hist_all [nh+1][max_ch+1],
 *     hist_quark (amplitude 1) [nh+1][2], hist_blip (amplitude <= nadir, other
 *     than 1) [nh+1][nadir+1], hist_spark [nh+1][max_ch+1]; column 0 of each is
 *     the class's trace count minus the other columns (:32-38);
 *   class_counts [3]: quarks, blips, sparks.
 * max_ch is the largest RyR count of a site (the reference has one count). */
casim_status casim_b200_release_analysis(casim_h h, double hist_dt_ms, double max_time_ms, int32_t nadir, double* per_site,
                                         int32_t* hist_all, int32_t* hist_quark, int32_t* hist_blip, int32_t* hist_spark,
                                         int32_t* class_counts);

/* Launch configuration chosen by measurement (no counterpart in the reference): on the
 * resident path, for every cluster-size class, candidate block sizes (256 up to the
 * specialisation's bound, step 64) at the class's cluster size and at twice it (where
 * the sites fit), and from 4 blocks on with even rows per block or with fewer rows on the
 * blocks that carry extra rim and deposit work, each run steps_per_trial time steps of that
 * class alone, from the same
 * state; the fastest is kept for later casim_b200_step calls. The batch state is the
 * same before and after. Later steps may differ from untuned ones in the last bits of
 * the cross-warp sums, and two tunings may choose differently. report (n bytes, may be
 * NULL) receives the choices. */
casim_status casim_b200_autotune(casim_h h, int64_t steps_per_trial, char* report, size_t n);

/* How the resident path splits the batch into thread-block-cluster classes,
 * or why the handle runs on the plain path. */
casim_status casim_b200_path_note(casim_h h, char* buf, size_t n);
/* Device timing of the last casim_b200_step call in milliseconds (CUDA events
 * recorded on the handle's stream around the launch sequence). */
casim_status casim_b200_last_step_ms(casim_h h, double* out);
/* Number of kernel launches issued by the last casim_b200_step call. */
casim_status casim_b200_last_step_launches(casim_h h, int64_t* out);
/* Per-site RyR gating models (no counterpart in the reference, whose runs have one
 * gating model): the sites listed gate by the two-state model of the "Dyad" /
 * "Channels" / "RyR" block of json_text (a Parameters.json of the reference's schema
 * naming the same ions; only its gating model is taken, spline tables and relative
 * file names resolved against base_dir); the other sites keep their model. Up to 7
 * models besides the handle's own; a later call moves the sites it lists again. For a
 * parameter sweep over gating laws in one batch: the model is a per-site choice inside
 * the warp-parallel gating kernel, everything else is shared. Served on the plain path
 * with its specialised kernels (create the handle with CASIM_PATH_PLAIN);
 * CASIM_EUNSUPPORTED on the resident path, for 60-state models, for layouts outside the
 * specialised kernels, and afterwards for the surrogate gating entry points. */
casim_status casim_b200_set_site_gating(casim_h h, const char* json_text, const char* base_dir, const int32_t* sites, int32_t n);
/* Profiling (no counterpart in the reference): advance every site by one time step
 * like casim_b200_step(h, 1) and return the device time in ms of each of its kernels,
 * from CUDA events on the handle's stream. Plain path: ms[0..3] = RyR gating and pools,
 * RD3D cytosol (0 without it), cleft stencil, Update; resident path: ms[0] = the one
 * launch. *count receives how many entries were written (at most n). Synchronous; not
 * while an open-RyR trace is enabled. */
casim_status casim_b200_profile_step(casim_h h, double* ms, int32_t n, int32_t* count);

/* Diagnostic: n runif() draws of the MRG32k3a stream with the given seed,
 * generated by a device kernel (the generator every site's gating uses).
 * Reproduces RngStream::RandU01 with incPrec = true (CaSim/rngstream.cpp:271-283).
 * A seed that RngStream's CheckSeed rejects (CaSim/rngstream.cpp:200-234) gives
 * CASIM_EINVAL. */
casim_status casim_b200_debug_rng(const uint32_t seed[6], int64_t n, double* out);

/* The generator of casim_b200_debug_rng for callers that cannot allocate
 * device memory (code inside another framework's memory pool, fixed-budget
 * real-time hosts, processes that must not grow their device footprint after
 * start-up). No counterpart in the reference. Its device staging buffer is a
 * fixed array of 262144 doubles (2 MiB) that every GPU loading the library
 * holds until exit; n above that is rejected with CASIM_EINVAL, and so is a
 * seed that RngStream's CheckSeed rejects (CaSim/rngstream.cpp:200-234). Calls
 * no allocator. Every call looks up the array's device address on the calling
 * thread's current device, launches on the legacy default stream and copies
 * the draws back synchronously, so no call may be made while a stream capture
 * is in progress on that device. All calls on a device share the array: calls
 * that overlap on the GPU race. out is host memory. */
casim_status casim_b200_rng_draws_static(const uint32_t seed[6], int64_t n, double* out);

/* ---- Quasi-stationary release sites: the reference's ParallelSolver path
 * (CaSim/ParallelSolver.cpp:51-143, CaSim/QuasyStationaryReleaseSite.cpp:89-133)
 * batched on the device, one scenario per warp. The mouth Ca of every RyR is the
 * background plus the linearised Naraghi-Neher increments of the open RyRs
 * (CaSim/LinearNaraghiNeher.cpp:9-75, computed on the host); gating is simulated
 * exactly with Gillespie's method (total rate, exponential waiting time, channel
 * picked by its share, its transition) until no RyR is open or "Max Time" is
 * reached. The JSON is the reference's ParallelSolver schema ("Calcium Release
 * Site" with "Parameters" / "Channels" / "Dyadic Cleft" / "Open Concentration");
 * two-state models (TwoStateMWC, TwoStateaHTG, SheepCannell), 1 to 1024 RyRs. seeds: 6 words per
 * scenario, or NULL for stream s of the package seed 12345 x 6; the streams carry on
 * from run to run. Each scenario keeps up to max_events events (time, channel, new
 * state). */
typedef struct casim_qs_s* casim_qs;
casim_status casim_b200_qs_create(const char* json_text, const char* base_dir, int32_t n_scenarios, const uint32_t* seeds,
                                  int64_t max_events, casim_qs* out);
casim_status casim_b200_qs_destroy(casim_qs h);
casim_status casim_b200_qs_last_error(casim_qs h, char* buf, size_t n);
casim_status casim_b200_qs_info(casim_qs h, int32_t* n_channels, int32_t* n_scenarios, double* max_time);
/* the increments [i][j]: Ca (uM) at RyR j from open RyR i (the "Open Concentration" at i itself) */
casim_status casim_b200_qs_increments(casim_qs h, double* out);
/* one run of every scenario, RyR first_channel[s] opened at t = 0
 * (CaSim/QuasyStationaryReleaseSite.cpp:92-98); synchronous. CASIM_EUNSUPPORTED when a
 * scenario had more events than max_events (its trace is truncated), CASIM_ETIMEOUT when
 * one was stopped after 64 x max_events events. */
casim_status casim_b200_qs_run(casim_qs h, const int32_t* first_channel);
casim_status casim_b200_qs_last_run_ms(casim_qs h, double* out);
/* events of the scenario's last run, stored or not (at most max_events are stored) */
casim_status casim_b200_qs_event_count(casim_qs h, int32_t scenario, int64_t* n);
/* the scenario's stored events in order: time (ms), channel, its new state (1 open);
 * min(event count, max_events) of them */
casim_status casim_b200_qs_events(casim_qs h, int32_t scenario, double* t, int32_t* channel, int32_t* state);
casim_status casim_b200_qs_draws(casim_qs h, int32_t scenario, uint64_t* out);
/* per scenario [5]: amplitude (most open RyRs), time to peak, time to end, integral of
 * the open count, its mean, and the class counts (quarks, blips up to nadir, sparks), as
 * IndChannelCREAnalyzer::RunAnalysis (CaSim/IndChannelCREAnalyzer.cpp:64-118). */
casim_status casim_b200_qs_analysis(casim_qs h, int32_t nadir, double* per_scenario, int32_t* class_counts);

/* ---- Surrogate of the quasi-steady Ca at the RyR mouths (no counterpart in
 * the reference; the plain RD step above generates its training snapshots and
 * judges its error). An MLP n_in -> depth x width (GELU) -> n_out with BF16
 * weights and activations and FP32 accumulation, every matrix product on the
 * tensor cores (tcgen05.mma), FP32 master weights updated by Adam. x, t and y
 * are DEVICE pointers to row-major FP32 [batch][n_in] / [batch][n_out];
 * batch must be a multiple of 128. width is 64, 128, 192 or 256; n_in <= 256,
 * n_out <= 256. */
typedef struct casim_surrogate_s* casim_sg;
casim_status casim_b200_sg_create(int n_in, int n_out, int width, int depth, uint64_t seed, casim_sg* out);
casim_status casim_b200_sg_destroy(casim_sg h);
casim_status casim_b200_sg_set_stream(casim_sg h, void* cuda_stream);
/* Parameter count: per layer W [dout][din] then b [dout], with din and dout
 * padded (n_in to a multiple of 64, n_out to a multiple of 128; padding is zero). */
casim_status casim_b200_sg_num_params(casim_sg h, int64_t* n);
/* FP32 parameters in the layout of casim_b200_sg_num_params (host memory). */
casim_status casim_b200_sg_get_params(casim_sg h, float* host);
casim_status casim_b200_sg_set_params(casim_sg h, const float* host);
/* y = net(x). */
casim_status casim_b200_sg_forward(casim_sg h, const float* x_dev, int batch, float* y_dev);
/* Mean-square loss over the n_out outputs and the gradient of every parameter
 * (host memory, parameter layout); no update. */
casim_status casim_b200_sg_gradients(casim_sg h, const float* x_dev, const float* t_dev, int batch, float* loss, float* grads_host);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on the mean-square loss; loss may be NULL. */
casim_status casim_b200_sg_train_step(casim_sg h, const float* x_dev, const float* t_dev, int batch, float lr, float* loss);
/* CASIM_ETIMEOUT if a tensor-core wait inside a kernel gave up. */
casim_status casim_b200_sg_check(casim_sg h);
/* Kernel launches issued by the handle so far. */
casim_status casim_b200_sg_launches(casim_sg h, int64_t* out);
casim_status casim_b200_sg_last_error(casim_sg h, char* buf, size_t n);
/* Surrogate-driven gating of a batch (casim_h). Features of every site into
 * x_dev [n_sites][ld] FP32 (device): per RyR slot (max_channels slots) its
 * open flag and grid position scaled to [-1, 1], then jSR Ca / 1000 uM, then
 * each dyad buffer total relative to its config value
 * (ld >= 3 max_channels + 1 + buffers). */
casim_status casim_b200_sg_features(casim_h h, int32_t max_channels, int32_t ld, float* x_dev);
/* Mouth Ca of every RyR = ca_ref * 10^y from the network output y_dev
 * [n_sites][ld] FP32 (device), RyR c of a site in column c. */
casim_status casim_b200_sg_set_mouth(casim_h h, const float* y_dev, int32_t ld, double ca_ref);
/* n time steps without the RD step (pool cytosol only): cytosol pool and jSR
 * ODEs, RyR gating (the draws of casim_b200_step) and RyR currents from the
 * mouth values held since casim_b200_sg_set_mouth. */
casim_status casim_b200_sg_gate_steps(casim_h h, int64_t n);
/* n surrogate-driven steps in windows of `window` steps, all on the batch's
 * stream with no host round trip: features, network (ca_ref * 10^output as
 * the mouth Ca of RyR slot c), casim_b200_sg_gate_steps(window). A full
 * window is captured once into a CUDA graph and replayed. Returns after the
 * stream is idle. A network handle serves one such call at a time. */
casim_status casim_b200_sg_run(casim_h h, casim_sg net, int32_t max_channels, int64_t n, int32_t window, double ca_ref);

/* Surrogate gating with periodic full-RD corrections and a residual fallback (no
 * counterpart in the reference). Time advances in periods of windows_per_check
 * windows of `window` steps, each period followed by rd_correction_steps steps of the
 * full RD method (the handle's path, gating included). After each correction the
 * network is evaluated on the current open sets and jSR and compared with the mouth
 * Ca the RD Update just produced: a site fails when the relative error at any of its
 * open RyRs' mouths exceeds tol. If more than max_fail_fraction of the sites fail, the next
 * period runs the full RD method instead of the surrogate (and is checked again
 * after its correction); otherwise it runs the surrogate. The RD fields do not move
 * during surrogate periods. stats (optional) counts the steps of each kind, the
 * checks and the fallbacks, and holds the last check's largest error and failing
 * fraction. */
typedef struct casim_sg_hybrid_stats {
    int64_t surrogate_steps, rd_steps, checks, fallbacks;
    double last_residual, last_fail_fraction;
} casim_sg_hybrid_stats;
casim_status casim_b200_sg_hybrid_run(casim_h h, casim_sg net, int32_t max_channels, int64_t n_steps, int32_t window,
                                      int32_t windows_per_check, int32_t rd_correction_steps, double tol, double max_fail_fraction,
                                      double ca_ref, casim_sg_hybrid_stats* stats);
/* One product C = A . B^T on the tensor cores: A [M][K] and B [N][K] BF16
 * (bit patterns), C [M][N] FP32, all device memory; M a multiple of 128,
 * N a multiple of 16 in [16, 256], K a multiple of 64. */
casim_status casim_b200_sg_gemm(const void* a_dev, const void* b_dev, int M, int N, int K, float* c_dev);

#ifdef __cplusplus
}
#endif
#endif
