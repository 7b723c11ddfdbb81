/* C entry points of the host engine: gsbn's Solver driven from C, Python
 * (ctypes) or any FFI, plus the format readers the tests check without a GPU.
 *
 * A solver is gsbn's Solver (src/gsbn/Solver.cpp:9-92): it reads a prototxt
 * network description, instantiates the procedures listed in its proc_param
 * entries through the procedure registry (ProcExtGen, ProcUpdLazy,
 * ProcExchangeSpike, ProcInitConn, ProcSpkRec, ProcCheck, ProcSnapshot) and
 * runs them until the stimulus schedule ends, writing the same record files.
 * gsbn_sim (src/gsbn_sim/Main.cpp:1-88) is a thin command line over these.
 *
 * Status codes are those of bcpnn.h; the message of the last failure on the
 * calling thread is returned by gsbn_engine_last_error().  Nothing throws
 * across this boundary.
 */
#ifndef GSBN_ENGINE_H
#define GSBN_ENGINE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gsbn_solver gsbn_solver;

#define GSBN_MODE_CPU 0
#define GSBN_MODE_GPU 1

/* Solver(NEW_SOLVER, net_path) when snapshot_path is NULL or empty, else
   Solver(COPY_SOLVER, net_path, snapshot_path) (Solver.cpp:9-65).  mode is
   GSBN_MODE_GPU; GSBN_MODE_CPU is accepted for interface parity and fails at
   the first tick (this build has no CPU path for ProcUpdLazy). */
int gsbn_solver_create(const char* net_path, const char* snapshot_path, int mode, gsbn_solver** out);

/* Solver::run (Solver.cpp:67-92).  windows != 0: one device run per stimulus
   segment when every listed procedure supports it; windows == 0: tick by
   tick through update_gpu, as gsbn's Upd does. */
int gsbn_solver_run(gsbn_solver* s, int windows);

/* ticks and windows run so far; the ProcCheck counts (-1 when not listed) */
int gsbn_solver_stats(const gsbn_solver* s, int64_t* ticks, int64_t* windows, int32_t* correct, int32_t* patterns);

/* the device network built by ProcUpdLazy (NULL before or without it), for
   bcpnn_read_state and friends */
int gsbn_solver_net(gsbn_solver* s, void** net);

int gsbn_solver_destroy(gsbn_solver* s);

/* message of the last failed call on this thread ("" if none) */
const char* gsbn_engine_last_error(void);

/* Parse a prototxt file and write its canonical dump (one field per line,
   defaults filled in) into out; *needed receives the size including the
   terminating NUL.  BCPNN_ERR_SIZE when cap is too small. */
int gsbn_prototxt_dump(const char* path, char* out, size_t cap, size_t* needed);

/* Decode a StimRawData file: dims = {data_rows, data_cols, mask_rows,
   mask_cols}; data/mask may be NULL to query the dimensions only. */
int gsbn_stim_decode(const char* path, uint32_t dims[4], uint32_t* data, size_t data_cap, float* mask, size_t mask_cap);

/* Names of the registered procedures, comma-separated. */
int gsbn_procedure_names(char* out, size_t cap);

#ifdef __cplusplus
}
#endif

#endif
