/* aoa_ckks.h — C ABI of the B200 CKKS evaluation engine (libaoa_b200.so).
 *
 * This is the drop-in boundary for the CKKS hot path of pdroalves/aoa
 * (aoa-ntt = library `newckks`, aoa-dgt = library `AOADGT`).  Every entry point
 * names the reference interface it replaces (paths relative to the reference
 * project root).  Plain pointers and sizes only; no C++ or torch types.
 *
 * Conventions
 *  - Every function returns an aoa_status; AOA_OK is 0.  A failed call leaves
 *    a message readable with aoa_last_error() (thread local).  Nothing exits
 *    the process (the reference's cudaCheckError() calls exit(1),
 *    aoa-ntt include/newckks/cuda/htrans/common.h:22-30).
 *  - Residues are uint64, limb-major: limb i of a polynomial is N consecutive
 *    words reduced modulo prime i.  Prime order is the Q primes (q_0..q_{k-1})
 *    then the special primes B (b_0..b_{kl-1}), as COPRIMES_BUCKET orders them
 *    (aoa-ntt src/cuda/manager.cu:426-564).
 *  - "Transform domain" is the reference's TRANSSTATE: position p holds the
 *    polynomial evaluated at psi^(2*bitrev(p)+1), psi = g^((q-1)/2N) with g the
 *    prime's smallest primitive root (the reference's PROOTS table).
 *  - All device work is asynchronous on the context's stream; aoa_ctx_sync
 *    waits for it.  One host thread per context (the reference's Context is not
 *    thread safe either, aoa-ntt include/newckks/tool/context.h:12-15).
 */
#ifndef AOA_CKKS_H
#define AOA_CKKS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  AOA_OK = 0,
  AOA_ERR_BAD_PARAM = 1,        /* invalid argument / unsupported parameters      */
  AOA_ERR_LEVEL_EXHAUSTED = 2,  /* level 0: reference throws (ckks.cpp:224-227)   */
  AOA_ERR_NO_KEY = 3,           /* missing switching key (e.g. rotation step)     */
  AOA_ERR_OOM = 4,              /* device allocation failed / over HBM budget     */
  AOA_ERR_CUDA = 5,             /* CUDA runtime error                             */
  AOA_ERR_TIMEOUT = 6,          /* bounded device wait expired                    */
  AOA_ERR_SLOT_MISMATCH = 7,    /* slots differ: reference throws (ckks.cpp:288)  */
  AOA_ERR_NOT_INITIALIZED = 8,
  AOA_ERR_NO_DEVICE = 9
} aoa_status;

/* Domain of a polynomial's residues (reference poly_states, defines.h:56-60):
 * coefficients (RNSSTATE), the negacyclic NTT domain of aoa-ntt (TRANSSTATE)
 * or the folded Gaussian-integer DGT domain of aoa-dgt (its TRANSSTATE).     */
typedef enum { AOA_COEF = 1, AOA_NTT = 2, AOA_DGT = 3 } aoa_domain;

typedef struct aoa_engine aoa_engine;
typedef struct aoa_ctx aoa_ctx;

typedef struct {
  int log_n;                  /* ring degree N = 2^log_n, 10 <= log_n <= 17        */
  int k;                      /* number of Q primes (levels 0..k-1)                */
  int kl;                     /* number of special primes for key switching       */
  const uint64_t* primes;     /* k + kl primes, each < 2^63, q = 1 mod 2N          */
  const uint64_t* generators; /* optional primitive roots (NULL: smallest root)    */
  int scale_bits;             /* default scale 2^scale_bits (cipher_init)          */
  int dnum;                   /* key-switching decomposition; must be 1            */
  const uint64_t* dgt_roots;  /* optional, 2 per prime: r = re + i im with r^(N/2) = i
                                 (the DGT twist root, aoa-dgt NTHROOT[p][N/2]); NULL:
                                 a root derived from the generator                  */
} aoa_params;

/* Last error message of this thread ("" if none). */
const char* aoa_last_error(void);
const char* aoa_status_string(int status);
/* Number of CUDA kernels this library has launched in this process (all
 * contexts); benchmarks difference it around a timed region.  No reference
 * counterpart (the reference has no launch accounting).                     */
long aoa_kernel_launches(void);

/* --- prime selection (host only, no device needed).  The reference picks its
 *     primes from fixed tables (src/cuda/htrans/coprimes.cu, selected by
 *     fill_ckks_coprimes_bucket, src/cuda/manager.cu:426-464) and their
 *     primitive roots from the PROOTS table.  aoa_search_primes returns the
 *     `count` largest primes of exactly `bits` bits with q = 1 mod `modulus`
 *     (descending; the count found is the return value, negative on error);
 *     aoa_primitive_root returns the smallest primitive root of prime q (the
 *     rule the reference's PROOTS entries follow), 0 if q is not prime.       */
int aoa_search_primes(int bits, uint64_t modulus, int count, uint64_t* out);
uint64_t aoa_primitive_root(uint64_t q);

/* --- engine: replaces CUDAManager::init / destroy
 *     (aoa-ntt include/newckks/cuda/manager.h:52-80, src/cuda/manager.cu:762-821)
 *     and NTTEngine::init (src/cuda/htrans/ntt.cu:750-1052).  Several engines may
 *     coexist (one per parameter set).  The engine binds the current device.   */
int aoa_engine_create(const aoa_params* params, aoa_engine** out);
int aoa_engine_destroy(aoa_engine* e);
/* Launch-shape knobs, no reference counterpart (its kernel shapes are
 * compile-time constants): "ntt_chunk_bytes" (bytes of limbs per transform
 * launch pair, default 4 GiB),
 * "ntt_waves" (transform CTAs per pass in resident waves, default 1),
 * "ntt_waves_large" (the same for launches of at least 1536 limbs, default 8),
 * "ntt_split" (log2 C - floor(log2 N / 2) of the R x C transform split,
 * -2..2, default 0), "dgt_split" (the same for the DGT's N/2-point cyclic
 * limb transforms, default 1), "ntt_cols_div" / "ntt_rows_div" (column-pass tile width
 * and row-pass tile height = widest >> div, 0..2, defaults 0 / 1),
 * "ntt_cols_kind" (0 CTA-wide exchange, 1 warp-owned columns; default 0),
 * "ntt_cols_tma" (1: the column pass loads 16-column tiles with one
 * tensor-map load, 0: one bulk copy per tile row; default 1),
 * "fuse" (bit mask of fused transform ends: 1 out-of-place inverse, 2 key
 * products, 4 key-switch combine; default 1), "batch_streams" (1 or 2
 * streams for a batched HMult group of 8 or more; default 2),
 * "conv_tensor_cores"
 * (0/1: basis conversion on the int8 tensor cores where it applies) and
 * "spin_limit" (polls of the kernels' bounded mbarrier waits before they
 * give up and report AOA_ERR_TIMEOUT at the next aoa_ctx_sync, 0..2^30;
 * default 2^20; the drain of copies and MMAs in flight after an expired
 * wait always uses the default bound).                                     */
int aoa_engine_tune(aoa_engine* e, const char* knob, double value);
/* current value of a knob (names as for aoa_engine_tune) */
int aoa_engine_tune_get(const aoa_engine* e, const char* knob, double* value);
/* Autotuner: times forward + inverse limb transforms of this engine's ring
 * over `limbs` limbs (0: about 1.5 GiB of limbs) and over batch-sized calls
 * (8 polys on each of two streams at once, scaled to the same limb count;
 * the sum is the objective, each figure the best of two timings) for
 * candidate splits, tile shapes, column-pass kinds, waves and chunk sizes
 * (coordinate descent from the current setting; a change is kept when it
 * is at least 2% faster), keeps the best and writes
 * a JSON report of the choice and the objective values (ms) into
 * report[0 .. report_len) (report may be NULL).  Run it before
 * the engine is used from other streams; it synchronises the device.       */
int aoa_engine_autotune(aoa_engine* e, int limbs, char* report, size_t report_len);
/* ring degree, prime count, primes (out may be NULL) */
int aoa_engine_info(const aoa_engine* e, int* log_n, int* k, int* kl, uint64_t* primes_out);

/* --- context: replaces Context (include/newckks/tool/context.h:16-49).
 *     stream == NULL creates a private stream.                                 */
int aoa_ctx_create(aoa_engine* e, void* cuda_stream, aoa_ctx** out);
int aoa_ctx_destroy(aoa_ctx* c);
/* Waits for the context's stream and reports device-side errors: a bounded
 * wait that expired in any kernel of the engine since the last report gives
 * AOA_ERR_TIMEOUT (and clears the record); the reference reports device
 * failures through cudaCheckError(), which exits the process
 * (include/newckks/cuda/htrans/common.h:20-29).                              */
int aoa_ctx_sync(aoa_ctx* c);
int aoa_ctx_stream(aoa_ctx* c, void** stream_out);
/* Check of the failure-detection path, no reference counterpart: launches on
 * the context's stream one kernel whose mbarrier wait can never complete (the
 * barrier expects an arrival that no thread, copy or MMA makes), with a limit
 * of `spins` polls; the wait runs out, the kernel records it in the engine's
 * error word exactly as the transform and conversion kernels do, and
 * returns with nothing in flight.  The next aoa_ctx_sync returns
 * AOA_ERR_TIMEOUT; the context stays usable.                                  */
int aoa_ctx_wait_check(aoa_ctx* c, int spins);

/* --- device memory on the context stream (poly_init / poly_copy_to_device /
 *     poly_copy_to_host, src/arithmetic/poly_t.cpp:10-100).                    */
int aoa_device_alloc(aoa_ctx* c, size_t bytes, void** out);
int aoa_device_free(aoa_ctx* c, void* p);
/* page-locked host memory, so host<->device copies run asynchronously */
int aoa_host_alloc(size_t bytes, void** out);
int aoa_host_free(void* p);
int aoa_memcpy_h2d(aoa_ctx* c, void* dst, const void* src, size_t bytes);
int aoa_memcpy_d2h(aoa_ctx* c, void* dst, const void* src, size_t bytes);
int aoa_memcpy_d2d(aoa_ctx* c, void* dst, const void* src, size_t bytes);

/* --- transforms: replace COMMONEngine::execute / NTTEngine::execute_ntt
 *     (src/cuda/htrans/common.cu:397-410, ntt.cu:463-475).  In place on device
 *     data laid out [npolys][poly_stride][N]; limbs 0..nlimbs-1 of each poly use
 *     primes first_prime..first_prime+nlimbs-1.                               */
int aoa_ntt_fwd(aoa_ctx* c, uint64_t* d_data, int npolys, int first_prime, int nlimbs, int poly_stride);
int aoa_ntt_inv(aoa_ctx* c, uint64_t* d_data, int npolys, int first_prime, int nlimbs, int poly_stride);

/* --- the DGT variant (aoa-dgt = library AOADGT).  A Gaussian-integer (GI)
 *     limb is N words, planar: the N/2 real parts then the N/2 imaginary parts
 *     of the folded polynomial a_j + i a_{j+N/2}, which is the same memory as
 *     the limb's N coefficients, so folding is free (poly_copy_to_device /
 *     poly_copy_to_host fold and unfold on the host, aoa-dgt
 *     src/arithmetic/polynomial.cu:92-154).
 *     aoa_dgt_fwd / aoa_dgt_inv replace DGTEngine::execute_dgt (aoa-dgt
 *     src/cuda/dgt.cu:1055-1096, kernels hdgt_tr/hidgt/hidgt_tr/dgt/idgt
 *     dgt.cu:805-1053): position p holds the folded polynomial at r w^bitrev(p),
 *     r the engine's twist root (aoa_params.dgt_roots), w = g^((q-1)/(N/2)).  */
int aoa_dgt_fwd(aoa_ctx* c, uint64_t* d_data, int npolys, int first_prime, int nlimbs, int poly_stride);
int aoa_dgt_inv(aoa_ctx* c, uint64_t* d_data, int npolys, int first_prime, int nlimbs, int poly_stride);
/* mul_dgt<GaussianInteger> (dgt.cu:1327-1341): element-wise GIMul (Karatsuba,
 * dgt.cu:530-553) of nlimbs transform-domain GI limbs, primes first_prime..  */
int aoa_gi_mul(aoa_ctx* c, uint64_t* d_out, const uint64_t* d_a, const uint64_t* d_b, int first_prime, int nlimbs);
/* The reference's GaussianInteger arrays ({re, im} pairs, [nlimbs][N/2]) to
 * planar GI limbs and back; no reference counterpart (the layout change the
 * planar format needs at the boundary).  Buffers must not overlap.          */
int aoa_gi_to_planar(aoa_ctx* c, uint64_t* d_dst, const uint64_t* d_src, int nlimbs);
int aoa_gi_from_planar(aoa_ctx* c, uint64_t* d_dst, const uint64_t* d_src, int nlimbs);
/* The engine's DGT twist roots, 2 words (re, im) per prime (compute_nthroot
 * inputs NTHROOT[p][N/2], dgt.cu:1612-1662).                                */
int aoa_engine_dgt_roots(const aoa_engine* e, uint64_t* roots_out);
/* Which library's transform the context's evaluations use: AOA_NTT (aoa-ntt,
 * default) or AOA_DGT (aoa-dgt: HMult tensor and key products as GIMul,
 * rotations through the coefficient domain).  Ciphertexts and keys carry
 * their domain; operands are converted on demand like poly_t states.  The
 * engine's DGT twist tables (12 words per prime and Gaussian integer) are
 * allocated by the first AOA_DGT setting or the first DGT of the engine.   */
int aoa_ctx_set_transform(aoa_ctx* c, int domain);

/* --- RNS basis conversion and rescale on device buffers (coefficient domain).
 *     aoa_modup replaces CUDAManager::execute_modup / fast_conv_Q_to_B_opt
 *     (src/cuda/manager.cu:180-249): reads Q limbs 0..level of in_q ([k][N]),
 *     writes the kl special limbs to out_b ([kl][N]).
 *     aoa_moddown replaces execute_moddown / fast_conv_B_to_Q
 *     (manager.cu:312-367): reads a QB poly ([k+kl][N]), writes limbs 0..level
 *     of out_q ([k][N]).
 *     aoa_rescale_polys replaces execute_rescale / ckks_rescale
 *     (manager.cu:90-139) on npolys polys of poly_stride limbs, in place.     */
int aoa_modup(aoa_ctx* c, const uint64_t* in_q, uint64_t* out_b, int level);
int aoa_moddown(aoa_ctx* c, const uint64_t* in_qb, uint64_t* out_q, int level);
int aoa_rescale_polys(aoa_ctx* c, uint64_t* d, int npolys, int poly_stride, int level);

/* --- ciphertexts: replace cipher_t / cipher_init / cipher_free
 *     (include/newckks/ckks/cipher_t.h:17-48, src/ckks/cipher_t.cpp:3-34).
 *     A ciphertext holds two polys of k limbs on the device; create sets
 *     level = k-1 and scale = 2^scale_bits like cipher_init.                  */
typedef struct aoa_ct aoa_ct;
int aoa_ct_create(aoa_ctx* c, aoa_ct** out);
int aoa_ct_destroy(aoa_ctx* c, aoa_ct* ct);
int aoa_ct_set(aoa_ct* ct, int level, int slots, uint64_t scale, int domain);
int aoa_ct_get(const aoa_ct* ct, int* level, int* slots, uint64_t* scale, int* domain);
int aoa_ct_data(aoa_ct* ct, uint64_t** device_ptr);          /* [2][k][N] */
/* host residues [2][nlimbs][N] (c0 then c1); upload sets level = nlimbs-1.
 * download converts a device copy to `domain` (poly_copy_to_host INTTs,
 * poly_t.cpp:74-100) and synchronises the stream.                           */
int aoa_ct_upload(aoa_ctx* c, aoa_ct* ct, const uint64_t* host, int nlimbs, int domain);
int aoa_ct_download(aoa_ctx* c, const aoa_ct* ct, uint64_t* host, int nlimbs, int domain);
/* aoa_ct_download queued without waiting (host pinned; read it after
 * aoa_ctx_sync): lets a caller overlap result copies with later work.     */
int aoa_ct_download_async(aoa_ctx* c, const aoa_ct* ct, uint64_t* host, int nlimbs, int domain);

/* --- switching keys: SwitchKey {a, b} over QB (include/newckks/defines.h:85-101,
 *     src/ckks/ckkskeys.cpp:101-191).  host_b / host_a: [k+kl][N] residues.   */
typedef struct aoa_swk aoa_swk;
int aoa_swk_create(aoa_ctx* c, const uint64_t* host_b, const uint64_t* host_a, int domain, aoa_swk** out);
int aoa_swk_destroy(aoa_ctx* c, aoa_swk* k);
/* device data [b | a], each (k+kl) limbs, and its transform domain */
int aoa_swk_data(aoa_swk* k, uint64_t** device_ptr, int* domain);
/* Key generation from given randomness (CKKSKeychain, src/ckks/ckkskeys.cpp:
 * 101-191, with the sampler's draws passed in), in the context's transform
 * domain.  Switching key for s1 under s2: b = rho(s1) + e - a s2, a over QB
 * (rho: ckks_rho, src/cuda/manager.cu:149-176; s1 NULL means 0).  d_s1, d_s2:
 * [k+kl][N] coefficient residues; d_a: [k+kl][N] uniform residues in a_domain;
 * d_e: N signed noise values.                                               */
int aoa_swk_generate(aoa_ctx* c, const uint64_t* d_s1, const uint64_t* d_s2, const uint64_t* d_a, int a_domain,
                     const int64_t* d_e, aoa_swk** out);
/* Public key (ckks_new_pk): out = (e - a s, a) over the Q primes, level k-1. */
int aoa_pk_generate(aoa_ctx* c, aoa_ct* out, const uint64_t* d_s, const uint64_t* d_a, int a_domain,
                    const int64_t* d_e);
/* Secrets of the evaluation, rotation and conjugation keys from s (nlimbs
 * coefficient-domain limbs): s^2 (ckks_new_mtk) and s(X^g) for odd g
 * (rotation by r: g = 5^r mod 2N; conjugation: g = 2N - 1).                  */
int aoa_secret_square(aoa_ctx* c, const uint64_t* d_s, uint64_t* d_out, int nlimbs);
int aoa_secret_galois(aoa_ctx* c, const uint64_t* d_s, uint64_t* d_out, long galois, int nlimbs);

/* --- CKKS evaluation (src/ckks/ckks.cpp; include/newckks/ckks/ckks.h:23-319).
 *     Outputs may alias inputs.  Like the reference, operands are brought to
 *     the domain an operation needs in place.                                 */
/* ckks_mul_without_rescale (ckks.cpp:273-332): out level = min level, scale =
 * floor(sa*sb/q_level), coefficient domain.                                  */
int aoa_hmult(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk);
/* ckks_mul (ckks.cpp:334-347): HMult + relinearise + rescale.                */
int aoa_hmult_relin_rescale(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk);
/* Batched ckks_mul / ckks_mul_without_rescale (rescale != 0 / == 0) of n
 * independent products out[i] = a[i] * b[i]: operands are grouped by level
 * and every stage of the pipeline runs as one launch over a group of up to 64
 * products.  No reference counterpart as one call (the reference runs the
 * products one ckks_mul at a time); results equal n separate calls.          */
int aoa_hmult_batch(aoa_ctx* c, int n, aoa_ct* const* out, aoa_ct* const* a, aoa_ct* const* b,
                    const aoa_swk* evk, int rescale);
/* The reference's per-call ckks_mul sequence (ckks.cpp:273-347 with the
 * poly_t.cpp domain rules: full-base transforms, unfused element-wise ops),
 * on this engine's kernels; same residues as aoa_hmult_relin_rescale, output
 * in coefficients.  The plain per-call baseline of the benchmarks.           */
int aoa_hmult_plain(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk);
/* The reference's per-call rotation and conjugation sequences
 * (ckks_rotate_left, ckks.cpp:982-1009, with rotate_slots_left,
 * encoder.cu:325-350; ckks_conjugate, ckks.cpp:1011-1040: the input back to
 * coefficients over the full base, the coefficient permutation, ModUp, whole-
 * QB transforms, unfused key products and ModDowns) on this engine's kernels;
 * same residues as aoa_rotate / aoa_conjugate, output in coefficients.  The
 * input keeps its domain (its inverse transform reads it out of place).  Steps
 * as in aoa_rotate.  The plain per-call baselines beside aoa_hmult_plain.    */
int aoa_rotate_plain(aoa_ctx* c, aoa_ct* out, aoa_ct* in, int steps, const aoa_swk* rtk);
int aoa_conjugate_plain(aoa_ctx* c, aoa_ct* out, aoa_ct* in, const aoa_swk* cjk);
/* HMult + relinearise + rescale that allocates nothing.  No counterpart in the
 * reference.  For callers that may not allocate device memory while they
 * evaluate (an application that owns the whole device memory budget through
 * its own allocator; a serving thread that cannot risk the device
 * synchronisation and driver lock of cudaMalloc / cudaFree): the same kernels
 * as aoa_hmult_relin_rescale, with their workspace in a fixed 32 MiB device
 * array built into the library (held by every device that loads it until the
 * process exits).  Parameter sets needing more workspace fail with
 * AOA_ERR_BAD_PARAM.  The first call in a CUDA context looks the array's
 * address up and caches it under that context (make it with the engine's
 * device current and before any stream capture; do not reset the device
 * between calls).  All calls share the one array: calls whose work overlaps
 * on the GPU race.                                                           */
int aoa_hmult_relin_rescale_noalloc(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk);
/* ckks_rescale (ckks.cpp:220-230) */
int aoa_rescale(aoa_ctx* c, aoa_ct* ct);
/* ckks_add / ckks_sub (ckks.cpp:232-271) */
int aoa_add(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b);
int aoa_sub(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b);
/* ckks_rotate_left (steps > 0) / ckks_rotate_right (steps < 0, i.e. left by
 * N/2 - |steps|) with the matching key (ckks.cpp:953-1009).                  */
int aoa_rotate(aoa_ctx* c, aoa_ct* out, aoa_ct* in, int steps, const aoa_swk* rtk);
/* n rotations by the same step with the same key (each op as aoa_rotate),
 * every stage one launch over the batch grouped by level; NTT contexts.    */
int aoa_rotate_batch(aoa_ctx* c, int n, aoa_ct* const* out, aoa_ct* const* in, int steps, const aoa_swk* rtk);
/* n rotations with a step and key per op (out[i] = in[i] rotated by
 * steps[i] with rtks[i], each as aoa_rotate): grouped by level only, so ops of
 * different steps share every launch of a group; NTT contexts.  No reference
 * counterpart as one call (the reference rotates one ciphertext per call). */
int aoa_rotate_batch_steps(aoa_ctx* c, int n, aoa_ct* const* out, aoa_ct* const* in, const int* steps,
                           const aoa_swk* const* rtks);
/* ckks_conjugate (ckks.cpp:1011-1040) */
int aoa_conjugate(aoa_ctx* c, aoa_ct* out, aoa_ct* in, const aoa_swk* cjk);
int aoa_conjugate_batch(aoa_ctx* c, int n, aoa_ct* const* out, aoa_ct* const* in, const aoa_swk* cjk);

/* --- CUDA-graph capture of a context's asynchronous work (no reference
 *     counterpart: the reference launches every kernel from the host).  Only
 *     asynchronous calls may sit between begin and end, after each work size
 *     has run once on the context (so nothing is allocated while capturing);
 *     a synchronising call ends the capture with an error.                    */
typedef struct aoa_graph aoa_graph;
int aoa_ctx_capture_begin(aoa_ctx* c);
int aoa_ctx_capture_end(aoa_ctx* c, aoa_graph** out);
int aoa_graph_launch(aoa_ctx* c, aoa_graph* g);
int aoa_graph_nodes(const aoa_graph* g, long* nodes);
int aoa_graph_destroy(aoa_graph* g);

/* --- plaintext / constant operations and slot sums (ckks.cpp:484-690).   */
/* ckks_mul / ckks_mul_without_rescale by an encoded plaintext (ckks.cpp:
 * 610-676): out = in * pt, scale = floor(in.scale * pt_scale / q_level),
 * rescaled when `rescale` != 0.  d_pt: [k][N] in pt_domain.                */
int aoa_mul_plaintext(aoa_ctx* c, aoa_ct* out, aoa_ct* in, const uint64_t* d_pt, int pt_domain, uint64_t pt_scale,
                      int rescale);
/* ckks_mul(_without_rescale) by a double (ckks.cpp:540-592): x = lrint(|val|
 * scale), negated for val < 0, scale = floor(scale^2 / q_level).            */
int aoa_mul_const(aoa_ctx* c, aoa_ct* out, aoa_ct* in, double val, int rescale);
/* ckks_add(ctx, c2, c1, double) (ckks.cpp:512-530): c0 +/- (uint64)(|val| scale). */
int aoa_add_const(aoa_ctx* c, aoa_ct* out, aoa_ct* in, double val);
/* ckks_sumslots (ckks.cpp:484-500): rotate-and-add over slots/2 .. 1;
 * rtks[j] is the left-rotation key for 2^j.                                */
int aoa_sumslots(aoa_ctx* c, aoa_ct* out, aoa_ct* in, const aoa_swk* const* rtks, int nkeys);
/* Compositions with the reference's operation sequences and metadata rules:
 * ckks_power (ckks.cpp:732-761; x = 0 gives the noiseless encryption of 1),
 * ckks_eval_polynomial (ckks.cpp:778-796, Horner from a cleared
 * accumulator), ckks_inner_prod of ciphertext pairs (ckks.cpp:423-441) and
 * with real weights (ckks.cpp:443-455).  out must differ from the input of
 * aoa_power / aoa_eval_polynomial.                                          */
int aoa_power(aoa_ctx* c, aoa_ct* out, aoa_ct* in, uint64_t x, const aoa_swk* evk);
int aoa_eval_polynomial(aoa_ctx* c, aoa_ct* out, aoa_ct* x, const double* coeffs, int n, const aoa_swk* evk);
int aoa_inner_prod(aoa_ctx* c, aoa_ct* out, aoa_ct* const* a, aoa_ct* const* b, int size, const aoa_swk* evk);
int aoa_inner_prod_const(aoa_ctx* c, aoa_ct* out, aoa_ct* const* a, const double* w, int size);

/* --- device samplers (Sampler, src/cuda/sampler.cu:13-230) on Philox4x32-10
 *     (Salmon et al., SC 2011): every draw is a function of (seed, stream,
 *     index), reproducible on the host.  Uniform residues of limbs
 *     first_prime .. +nlimbs ([nlimbs][N], 128-bit draw mod q); rounded
 *     Gaussian (Box-Muller, sigma); ternary with exactly hw entries +-1
 *     (sample_hw: hw = 64, sample_Z0: hw = N/2).  Asynchronous.             */
int aoa_sample_uniform(aoa_ctx* c, uint64_t* d_out, int first_prime, int nlimbs, uint64_t seed, uint64_t stream);
int aoa_sample_gaussian(aoa_ctx* c, int64_t* d_out, long n, double sigma, uint64_t seed, uint64_t stream);
int aoa_sample_ternary(aoa_ctx* c, int64_t* d_out, long n, long hw, uint64_t seed, uint64_t stream);
/* small signed integers (N of them) -> [nlimbs][N] canonical residues */
int aoa_signed_to_residues(aoa_ctx* c, const int64_t* d_in, uint64_t* d_out, int first_prime, int nlimbs);

/* --- binary wire format (serving payloads; the reference's JSON export,
 *     cipher_export / cipher_import cipher_t.cpp:42-81 and export_keys /
 *     load_keys ckkscontext.cpp:50-100, is in the Python package).  A 64-byte
 *     header (magic "AOACKKS1", kind, ring, primes fingerprint, level, slots,
 *     scale, domain) and the residues as u64: a ciphertext's live limbs in its
 *     current domain, a key's two (k+kl)-limb polys.  Readers reject buffers
 *     of another kind, ring, prime set or length (AOA_ERR_BAD_PARAM).        */
size_t aoa_ct_wire_size(const aoa_ctx* c, const aoa_ct* ct);
int aoa_ct_serialize(aoa_ctx* c, const aoa_ct* ct, uint8_t* buf, size_t cap, size_t* len);
int aoa_ct_deserialize(aoa_ctx* c, aoa_ct* ct, const uint8_t* buf, size_t len);
size_t aoa_swk_wire_size(const aoa_ctx* c);
int aoa_swk_serialize(aoa_ctx* c, const aoa_swk* k, uint8_t* buf, size_t cap, size_t* len);
int aoa_swk_deserialize(aoa_ctx* c, const uint8_t* buf, size_t len, aoa_swk** out);

/* --- encoder and encryption (src/ckks/encoder.cu:12-298, ckks.cpp:87-192,
 *     CKKSContext::encode/decode ckkscontext.cpp:5-38).  Complex values are
 *     (re, im) double pairs (the layout of std::complex<double>).             */
/* ckks_encode (encoder.cu:166-221): `filled` values then `empty` zero slots
 * (filled + empty a power of two <= N/2), scaled by `scale`, into limbs
 * 0..nlimbs-1 of d_out ([nlimbs][N]) in `domain`.  Identical residues.        */
int aoa_encode(aoa_ctx* c, const double* host_vals, int filled, int empty, uint64_t scale, int nlimbs,
               int domain, uint64_t* d_out);
/* CKKSContext::decode + ckks_decode (ckkscontext.cpp:21-38, encoder.cu:259-298):
 * `slots` values from limb 0 of d_m (in `domain`) into host memory; identical
 * doubles.  Synchronises.                                                    */
int aoa_decode(aoa_ctx* c, const uint64_t* d_m, int domain, int slots, uint64_t scale, double* host_vals);
/* ckks_encrypt_poly (ckks.cpp:87-105) with the sampler's draws passed in:
 * d_u, d_e1, d_e2 hold N signed coefficients each (the Z0 and DG samples);
 * pk = (b, a) as a ciphertext over all Q primes.  d_m: [k][N] message in
 * m_domain.  Output in the NTT domain at level k-1.                          */
int aoa_encrypt(aoa_ctx* c, aoa_ct* out, const uint64_t* d_m, int m_domain, aoa_ct* pk, const int64_t* d_u,
                const int64_t* d_e1, const int64_t* d_e2, int slots, uint64_t scale);
/* ckks_decrypt_poly (ckks.cpp:179-192): m = c1 s + c0 over limbs 0..level,
 * coefficient domain, into d_m_out ([level+1][N]).  d_s: [k][N] secret.     */
int aoa_decrypt(aoa_ctx* c, aoa_ct* ct, const uint64_t* d_s, int s_domain, uint64_t* d_m_out);

#ifdef __cplusplus
}
#endif
#endif /* AOA_CKKS_H */
