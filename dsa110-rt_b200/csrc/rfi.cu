// RFI excision by voltage zero-fill on the raw on-wire pages (sm_100a):
// apply_rfi_mask_to_voltages (src/dsart/services/corr_fast_integration.py:
// 1249-1370) moved ahead of the unpack.  A byte of a page (npkt, nant,
// nchan, 2t, 2p) is one complex 4-bit sample; a flagged sample becomes 0,
// both nibbles zero, which is the voltage 0 + 0i the reference writes after
// its unpack.  So the correlator never sees it.
//
// Flags (True == flagged, one byte each):
//   mask      (n_pages, nant, nchan, 2pol), per (antenna, channel, pol);
//   time_mask (n_pages, n_acc, nchan, 2pol), per accumulation of npkt/n_acc
//             packets, on every antenna.
// One CTA per (packet, page); a thread takes the 4-byte words (two times x
// two pols) of its (antenna, channel) cells and writes only flagged ones.
#include "dsb_common.cuh"

namespace {

int launch_status() { return cudaGetLastError() == cudaSuccess ? DSB_OK : DSB_E_CUDA; }

__global__ void __launch_bounds__(256) rfi_zero_fill_kernel(
    uint32_t* __restrict__ raw, int npkt, int nant, int nchan,
    const uint8_t* __restrict__ mask, const uint8_t* __restrict__ time_mask, int n_acc) {
  const int pkt = blockIdx.x, page = blockIdx.y;
  const int cells = nant * nchan;
  uint32_t* row = raw + ((long long)page * npkt + pkt) * cells;
  const uint8_t* tm = time_mask
      ? time_mask + ((long long)page * n_acc + pkt / (npkt / n_acc)) * nchan * 2
      : nullptr;
  const uint8_t* am = mask ? mask + (long long)page * cells * 2 : nullptr;
  for (int i = threadIdx.x; i < cells; i += blockDim.x) {
    const int ch = i % nchan;
    bool f0 = false, f1 = false;
    if (am) {
      f0 = am[2 * i] != 0;
      f1 = am[2 * i + 1] != 0;
    }
    if (tm) {
      f0 = f0 || tm[2 * ch] != 0;
      f1 = f1 || tm[2 * ch + 1] != 0;
    }
    // bytes of a word: (t0,p0) (t0,p1) (t1,p0) (t1,p1), low byte first
    if (f0 || f1) row[i] &= (f0 ? 0u : 0x00ff00ffu) | (f1 ? 0u : 0xff00ff00u);
  }
}

}  // namespace

extern "C" {

int dsb_rfi_zero_fill(void* raw, int n_pages, int npkt, int nant, int nchan,
                      const unsigned char* mask, const unsigned char* time_mask, int n_acc,
                      cudaStream_t stream) {
  if (!raw || n_pages < 0 || npkt < 0 || nant <= 0 || nchan <= 0) return DSB_E_ARG;
  if (time_mask && (n_acc <= 0 || npkt % n_acc != 0)) return DSB_E_ARG;
  if (reinterpret_cast<uintptr_t>(raw) & 3) return DSB_E_ARG;
  if (n_pages == 0 || npkt == 0 || (!mask && !time_mask)) return DSB_OK;
  if (n_pages > 65535) return DSB_E_CAPACITY;
  dim3 grid(npkt, n_pages);
  rfi_zero_fill_kernel<<<grid, 256, 0, stream>>>((uint32_t*)raw, npkt, nant, nchan, mask,
                                                 time_mask, n_acc);
  return launch_status();
}

}  // extern "C"
