// sp_dev_internal.h -- layout of the device state of one reservoir (CUDA side
// only; the host C code sees sp_dev as an opaque type).
//
// HBM layout (n neurons, L ring rows, nw = ceil(n/32) spike words):
//   V[n], tprev[n]                   membrane potential, refractory clock
//   ring[L][n]   (FLIF_GL)           time-major history: lag k of every neuron
//                                    is one contiguous n*8-byte row
//   ring[n][D]   (FLIF_CAPUTO)       per-neuron shift register (own head)
//   spk[2][nw]                       spike bits, double-buffered per micro-step
//   row_ptr[n+1] (int64), col[nnz] (int32), w[nnz] (double)   recurrent CSR
//   eff[2][n]                        per-neuron synaptic drive (non-SIMPLE)
//   Iring[Ls][n] (FRACTIONAL)        time-major fractional-current ring
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <vector>
#include "sp_dev.h"

struct sp_dev {
    int device, num_sms, coop;
    int l2_bytes;  // device L2 cache size
    int l2_hinted; // a launch read the ring with evict-last hints (demoted at destroy)
    cudaStream_t stream;
    int n, din, dout, micro;
    int nw;              // warps of positions (= spike words in position space)
    int rs;              // positions = 32 * nw (device arrays are in position order)
    size_t ring_elems;
    size_t nwords, nnz;  // nwords = nw (position-space spike words)
    size_t nwords_nat;   // spike words of a neuron-order raster, ceil(n / 32)
    int bal_G;           // layout balanced over this many CTAs (0: dense layout)
    double dt, gamma;
    int ntype, stype;
    sp_neuron_consts nc;
    sp_synapse_consts sc;
    unsigned long long seed;
    long long step;      // neuron micro-step counter (reset -> 0)
    long long syn_step;  // fractional-synapse micro-step counter (never reset)
    int phase;           // spk buffer holding the latest spike words
    long long launches;
    sp_launch launch;

    double *V, *tprev, *ring;
    int *cap_pos;
    long long *refr_until;
    unsigned long long *rng;
    unsigned *spk;
    long long *row_ptr;
    int *col;
    double *w, *coef;
    double *eff, *trace, *edge_decay, *edge_omd, *edge_trace;
    double *scoef, *Iring;
    double *mx_decay, *mx_omd, *mx_c, *mx_tr;
    double *W_in, *W_out;  // rows / columns in position order
    long long *h_row_ptr;  // host copy of row_ptr [rs + 1] (launch planning)
    int *pos_of;           // [n] position of neuron i
    int *nid_of;           // [rs] neuron at position q, or -1

    // staging for host-driven runs
    size_t chunk;        // macro steps per chunk
    double *d_u;         // [chunk][din]
    double *d_phi;       // [chunk][rs] position-space states
    double *d_nat;       // [chunk][n] neuron-order states
    double *d_y;         // [chunk][dout]
    unsigned *d_ras;     // [chunk][nw] position-space spike words
    unsigned *d_ras_nat; // [chunk][nw] neuron-order spike words
    double *d_spkd;      // [n]
    double *h_stage;     // pinned [chunk][dout]
    unsigned long long *bar;  // grid-barrier arrival counter
    unsigned long long *flags; // per-CTA arrival flags of the step kernel (flag_cap CTAs)
    int flag_cap;
    int *err;                 // [0] code, [1]/[2] micro-step low/high word

    // bounded waits: limit (ns) of every wait in the step kernel; one-shot
    // test hook (CTA hold_cta withholds its arrival at micro-step hold_b of
    // the next launch, -1 = none); the last device error seen by the host
    unsigned long long wait_ns;
    int hold_cta;
    long long hold_b;
    int last_err_code;
    long long last_err_step;

    // 2-D tiled tensor map over the FLIF_GL ring (variant 1), box BW x R
    CUtensorMap tmap;
    int tmap_bw, tmap_r;
};

extern "C" int sp_dev_launch_chunk(sp_dev *d, const double *u, size_t T, double *phi,
                                   unsigned *raster);
extern "C" int sp_dev_readout(sp_dev *d, const double *X, size_t T, double *Y);
extern "C" void sp_dev_note_error(const char *what, int code);
extern "C" int sp_dev_gather_rows(sp_dev *d, const double *pos_rows, size_t T, double *nat_rows);
extern "C" int sp_dev_w_out_from_nat(sp_dev *d, const double *dev_w_nat);
extern "C" int sp_dev_w_out_to_nat(sp_dev *d, double *dev_w_nat);

// Position layout shared by the single and batched paths (dev_reservoir.cu).
void sp_make_layout(const sp_host_model *m, int nw, const std::vector<int> *cap,
                    std::vector<int> &pos_of,
                    std::vector<int> &nid_of);

// Ridge on a device Phi [T x n] (neuron order) and targets Y [T x dout];
// writes d_W_out [dout x n] or returns SP_RIDGE_SINGULAR (dev_readout.cu).
extern "C" int sp_ridge_phi(cudaStream_t s, const double *Phi, int n, size_t T,
                            const double *Y, int dout, double lambda, const sp_ridge_opts *o,
                            sp_ridge_report *rep, double *d_W_out);
// The same with reusable work buffers (primal solves of up to 16 outputs).
struct sp_ridge_ws;
extern "C" sp_ridge_ws *sp_ridge_ws_new(void);
extern "C" void sp_ridge_ws_free(sp_ridge_ws *w);
extern "C" int sp_ridge_phi_ws(cudaStream_t s, const double *Phi, int n, size_t T,
                               const double *Y, int dout, double lambda, const sp_ridge_opts *o,
                               sp_ridge_report *rep, double *d_W_out, sp_ridge_ws *ws);

// Layout kernels on raw device pointers (dev_reservoir.cu).
extern "C" int sp_launch_readout(cudaStream_t s, const double *W_pos, const double *X, int rs,
                                 size_t T, int dout, double *Y);
extern "C" int sp_launch_gather_rows(cudaStream_t s, const double *pos_rows, int rs,
                                     const int *pos_of, int n, size_t T, double *nat_rows);
extern "C" int sp_launch_wout_to_pos(cudaStream_t s, const double *w_nat, const int *nid_of, int n,
                                     int rs, int dout, double *w_pos);
