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

/* Domain of a polynomial's residues (reference poly_states, defines.h:56-60). */
typedef enum { AOA_COEF = 1, AOA_NTT = 2 } aoa_domain;

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
} aoa_params;

/* Last error message of this thread ("" if none). */
const char* aoa_last_error(void);
const char* aoa_status_string(int status);

/* --- engine: replaces CUDAManager::init / destroy
 *     (aoa-ntt include/newckks/cuda/manager.h:52-80, src/cuda/manager.cu:762-821)
 *     and NTTEngine::init (src/cuda/htrans/ntt.cu:750-1052).  Several engines may
 *     coexist (one per parameter set).  The engine binds the current device.   */
int aoa_engine_create(const aoa_params* params, aoa_engine** out);
int aoa_engine_destroy(aoa_engine* e);
/* ring degree, prime count, primes (out may be NULL) */
int aoa_engine_info(const aoa_engine* e, int* log_n, int* k, int* kl, uint64_t* primes_out);

/* --- context: replaces Context (include/newckks/tool/context.h:16-49).
 *     stream == NULL creates a private stream.                                 */
int aoa_ctx_create(aoa_engine* e, void* cuda_stream, aoa_ctx** out);
int aoa_ctx_destroy(aoa_ctx* c);
int aoa_ctx_sync(aoa_ctx* c);
int aoa_ctx_stream(aoa_ctx* c, void** stream_out);

/* --- device memory on the context stream (poly_init / poly_copy_to_device /
 *     poly_copy_to_host, src/arithmetic/poly_t.cpp:10-100).                    */
int aoa_device_alloc(aoa_ctx* c, size_t bytes, void** out);
int aoa_device_free(aoa_ctx* c, void* p);
int aoa_memcpy_h2d(aoa_ctx* c, void* dst, const void* src, size_t bytes);
int aoa_memcpy_d2h(aoa_ctx* c, void* dst, const void* src, size_t bytes);
int aoa_memcpy_d2d(aoa_ctx* c, void* dst, const void* src, size_t bytes);

/* --- transforms: replace COMMONEngine::execute / NTTEngine::execute_ntt
 *     (src/cuda/htrans/common.cu:397-410, ntt.cu:463-475).  In place on device
 *     data laid out [npolys][poly_stride][N]; limbs 0..nlimbs-1 of each poly use
 *     primes first_prime..first_prime+nlimbs-1.                               */
int aoa_ntt_fwd(aoa_ctx* c, uint64_t* d_data, int npolys, int first_prime, int nlimbs, int poly_stride);
int aoa_ntt_inv(aoa_ctx* c, uint64_t* d_data, int npolys, int first_prime, int nlimbs, int poly_stride);

#ifdef __cplusplus
}
#endif
#endif /* AOA_CKKS_H */
