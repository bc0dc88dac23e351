// Native continuous-batching loop for mixed-size detection requests (host code; no reference counterpart).
//
// The lanes and their captured graphs are built by arpeggio_b200.serve.Server (one detector per lane, a graph per
// power-of-two batch size that runs the chain on the lane's device buffers); this loop only admits, copies the
// requests in (straight from the streams' host arrays), replays, copies the results out (straight into the streams'
// output rows) and polls, so the polling path has neither the interpreter nor host-side copies of the data.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "../../include/arpeggio_b200.h"

namespace {

constexpr int kMaxGraphs = 32;

struct LaneState {
  cudaEvent_t ev = nullptr;
  int maxk = 0;         // the largest batch with a graph
  bool busy = false;
  int a = 0, b = 0;     // request rows in flight
};

bool stream_ok(const arp_serve_stream& s) {
  if (s.n < 0 || s.h_elems <= 0 || s.y_elems <= 0 || s.bits_per <= 0) return false;
  return s.n == 0 || (s.H && s.y && s.s2 && s.snr && s.rid && s.t_arrival && s.bits && s.dist && s.done);
}

}  // namespace

extern "C" int arp_serve_run(const arp_serve_stream* streams, int nstreams, const arp_serve_lane* lanes, int nlanes,
                             double timeout_s, int64_t* batches) {
  if (nstreams < 0 || nlanes < 0 || (nstreams > 0 && !streams) || (nlanes > 0 && !lanes)) return ARP_ERR_ARG;
  for (int s = 0; s < nstreams; ++s)
    if (!stream_ok(streams[s])) return ARP_ERR_ARG;
  std::vector<LaneState> st(nlanes);
  std::vector<std::vector<int>> lanes_of(nstreams);
  for (int l = 0; l < nlanes; ++l) {
    const arp_serve_lane& ln = lanes[l];
    if (ln.cls < 0 || ln.cls >= nstreams || !ln.Hd || !ln.yd || !ln.s2d || !ln.snrd || !ln.instd || !ln.bitsd ||
        !ln.distd || ln.ngraphs < 1 || ln.ngraphs > kMaxGraphs)
      return ARP_ERR_ARG;
    for (int i = 0; i < ln.ngraphs; ++i)
      if (!ln.graphs[i] || ln.sizes[i] < 1 || (i > 0 && ln.sizes[i] <= ln.sizes[i - 1])) return ARP_ERR_ARG;
    st[l].maxk = ln.sizes[ln.ngraphs - 1];
    lanes_of[ln.cls].push_back(l);
  }
  for (int s = 0; s < nstreams; ++s)
    if (streams[s].n > 0 && lanes_of[s].empty()) return ARP_ERR_ARG;  // requests no lane can take
  for (int l = 0; l < nlanes; ++l) {
    if (cudaEventCreateWithFlags(&st[l].ev, cudaEventDisableTiming) != cudaSuccess) {
      for (int j = 0; j < l; ++j) cudaEventDestroy(st[j].ev);
      return ARP_ERR_LAUNCH;
    }
  }
  if (batches)
    for (int s = 0; s < nstreams; ++s) batches[s] = 0;
  std::vector<int> next(nstreams, 0);
  const auto t0 = std::chrono::steady_clock::now();
  auto clock = [&t0]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
  int rc = ARP_OK;
  for (;;) {
    const double now = clock();
    long long left = 0;
    // completions: a lane whose batch is done hands its results over and becomes free
    for (int l = 0; l < nlanes && rc == ARP_OK; ++l) {
      LaneState& ls = st[l];
      if (!ls.busy) continue;
      const cudaError_t q = cudaEventQuery(ls.ev);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) {
        rc = ARP_ERR_LAUNCH;
        break;
      }
      const arp_serve_stream& s = streams[lanes[l].cls];  // its results are already in the output rows
      for (int r = ls.a; r < ls.b; ++r) s.done[r] = now;
      ls.busy = false;
    }
    if (rc != ARP_OK) break;
    // admissions: a free lane takes what has arrived, up to its largest graph
    for (int c = 0; c < nstreams && rc == ARP_OK; ++c) {
      const arp_serve_stream& s = streams[c];
      const int arrived = (int)(std::upper_bound(s.t_arrival, s.t_arrival + s.n, now) - s.t_arrival);
      for (int l : lanes_of[c]) {
        LaneState& ls = st[l];
        if (ls.busy || next[c] >= arrived) continue;
        const arp_serve_lane& ln = lanes[l];
        const int a = next[c], k = std::min(arrived - a, ls.maxk);
        int g = 0;
        while (ln.sizes[g] < k) ++g;  // the smallest graph that holds the batch
        const cudaStream_t cs = static_cast<cudaStream_t>(ln.stream);
        const cudaMemcpyKind in = cudaMemcpyHostToDevice, out = cudaMemcpyDeviceToHost;
        if (cudaMemcpyAsync(ln.Hd, s.H + (size_t)a * s.h_elems, (size_t)k * s.h_elems * sizeof(float), in, cs) ||
            cudaMemcpyAsync(ln.yd, s.y + (size_t)a * s.y_elems, (size_t)k * s.y_elems * sizeof(float), in, cs) ||
            cudaMemcpyAsync(ln.s2d, s.s2 + a, (size_t)k * sizeof(float), in, cs) ||
            cudaMemcpyAsync(ln.snrd, s.snr + a, (size_t)k * sizeof(float), in, cs) ||
            cudaMemcpyAsync(ln.instd, s.rid + a, (size_t)k * sizeof(int32_t), in, cs) ||
            cudaGraphLaunch(static_cast<cudaGraphExec_t>(ln.graphs[g]), cs) ||
            cudaMemcpyAsync(s.bits + (size_t)a * s.bits_per, ln.bitsd, (size_t)k * s.bits_per, out, cs) ||
            cudaMemcpyAsync(s.dist + a, ln.distd, (size_t)k * sizeof(float), out, cs) ||
            cudaEventRecord(ls.ev, cs)) {
          rc = ARP_ERR_LAUNCH;
          break;
        }
        ls.busy = true;
        ls.a = a;
        ls.b = a + k;
        next[c] = a + k;
        if (batches) ++batches[c];
      }
      left += s.n - next[c];
    }
    for (int l = 0; l < nlanes; ++l) left += st[l].busy ? 1 : 0;
    if (rc != ARP_OK || left == 0) break;
    if (now > timeout_s) {
      rc = ARP_ERR_TIMEOUT;
      break;
    }
  }
  // batches still in flight finish before the caller reads the outputs or reuses the lanes (their kernels' waits
  // are bounded)
  for (int l = 0; l < nlanes; ++l) {
    if (st[l].busy) cudaEventSynchronize(st[l].ev);
    cudaEventDestroy(st[l].ev);
  }
  return rc;
}
