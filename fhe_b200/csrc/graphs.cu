// CUDA-graph replay of multi-kernel engine operations.  A bootstrap launches
// thousands of kernels and a serving batch hundreds per ciphertext; once an
// operation's shape has run directly (which checks its inputs and builds every
// table it needs), it is captured once on the engine's stream, temporaries
// allocated and freed inside the graph, and replayed from then on: one launch per
// call, the same kernels and the same words.  The items of a batch run on several
// streams (forked from and joined into the engine's stream), so one item's kernels
// fill the SMs that another's last wave of CTAs leaves idle; captured, the items
// become parallel branches of the graph.
#include <algorithm>
#include <cstring>

#include "engine.hpp"

namespace fhe_b200 {

namespace {

uint64_t double_bits(double x) {
  uint64_t u;
  std::memcpy(&u, &x, sizeof(u));
  return u;
}

}  // namespace

std::vector<std::unique_ptr<Data>> Engine::run_captured(std::vector<uint64_t> key,
                                                        const std::vector<const Data *> &inputs,
                                                        const GraphBody &body) {
  if (!graphs_ || profiling_) return body(inputs);
  key.insert(key.end(), {static_cast<uint64_t>(tensor_cores_), static_cast<uint64_t>(fused_bsgs_),
                         static_cast<uint64_t>(value_transforms_)});
  for (const Data *d : inputs) {
    const double hi = static_cast<double>(d->scale);
    key.insert(key.end(), {static_cast<uint64_t>(d->type), static_cast<uint64_t>(d->flag),
                           static_cast<uint64_t>(d->moduli_id), static_cast<uint64_t>(d->polys),
                           double_bits(hi),
                           double_bits(static_cast<double>(d->scale - static_cast<long double>(hi)))});
  }
  key.push_back(reinterpret_cast<uint64_t>(stream_));
  if (graph_failed_.count(key)) return body(inputs);

  auto seen = graph_seen_.find(key);
  if (seen == graph_seen_.end()) {
    auto out = body(inputs);
    std::vector<GraphShape> shapes;
    for (const auto &o : out) shapes.push_back({o->type, o->flag, o->moduli_id, o->polys, o->scale});
    graph_seen_[key] = shapes;
    return out;
  }

  auto it = graph_cache_.find(key);
  if (it == graph_cache_.end()) {
    CapturedGraph g;
    std::vector<const Data *> private_in;
    for (const Data *d : inputs) {
      g.in.push_back(make_data(d->type, d->flag, d->moduli_id, d->polys, d->scale));
      g.in.back()->delta = d->delta;
      private_in.push_back(g.in.back().get());
    }
    for (const GraphShape &s : seen->second)
      g.out.push_back(make_data(s.type, s.flag, s.moduli_id, s.polys, s.scale));
    synchronize();  // the graph's inputs and outputs exist before the capture starts
    cudaGraph_t graph = nullptr;
    check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
    const unsigned long long counted = kernel_launch_count();
    cudaError_t e = cudaSuccess;
    try {
      auto out = body(private_in);
      if (out.size() != g.out.size()) e = cudaErrorInvalidValue;
      for (size_t i = 0; e == cudaSuccess && i < out.size(); i++) {
        if (out[i]->words() != g.out[i]->words()) {
          e = cudaErrorInvalidValue;
          break;
        }
        e = cudaMemcpyAsync(g.out[i]->d, out[i]->d, out[i]->words() * sizeof(int64_t),
                            cudaMemcpyDeviceToDevice, stream_);
      }
    } catch (...) {
      e = cudaErrorStreamCaptureInvalidated;
    }
    const cudaError_t end = cudaStreamEndCapture(stream_, &graph);
    g.launches = kernel_launch_count() - counted;
    unnote_launches(g.launches);  // nothing ran during the capture
    if (e == cudaSuccess) e = end;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      // Something on the path cannot be captured: keep running it directly.
      cudaGetLastError();
      graph_failed_.insert(key);
      return body(inputs);
    }
    it = graph_cache_.emplace(key, std::move(g)).first;
  }

  CapturedGraph &g = it->second;
  for (size_t i = 0; i < inputs.size(); i++)
    check(cudaMemcpyAsync(g.in[i]->d, inputs[i]->d, inputs[i]->words() * sizeof(int64_t),
                          cudaMemcpyDeviceToDevice, stream_),
          "graph input");
  check(cudaGraphLaunch(g.exec, stream_), "graph launch");
  note_launch(static_cast<unsigned>(g.launches));
  std::vector<std::unique_ptr<Data>> out;
  for (const auto &o : g.out) out.push_back(clone(*o));
  return out;
}

void Engine::set_concurrency(int streams) {
  if (streams < 1 || streams > kMaxConcurrency)
    throw std::invalid_argument("set_concurrency: the stream count should be between 1 and 8.");
  if (!fork_) check(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "cudaEventCreate");
  while (static_cast<int>(workers_.size()) < streams) {
    cudaStream_t w = nullptr;
    check(cudaStreamCreateWithFlags(&w, cudaStreamNonBlocking), "cudaStreamCreate");
    workers_.push_back(w);
    cudaEvent_t ev = nullptr;
    check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
    worker_done_.push_back(ev);
  }
  concurrency_ = streams;
}

void Engine::run_concurrent(int count, const std::function<void(int)> &item) {
  const int streams = std::min(count, concurrency_);
  if (streams <= 1) {
    for (int i = 0; i < count; i++) item(i);
    return;
  }
  // Inside a capture of the engine's stream the fork and join events make the
  // workers part of the same graph, as parallel branches.
  const cudaStream_t home = stream_;
  check(cudaEventRecord(fork_, home), "fork");
  for (int w = 0; w < streams; w++) check(cudaStreamWaitEvent(workers_[w], fork_, 0), "fork");
  auto join = [&] {
    stream_ = home;
    cudaError_t e = cudaSuccess;
    for (int w = 0; w < streams; w++) {
      if (e == cudaSuccess) e = cudaEventRecord(worker_done_[w], workers_[w]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(home, worker_done_[w], 0);
    }
    return e;
  };
  try {
    for (int i = 0; i < count; i++) {
      stream_ = workers_[i % streams];
      item(i);
    }
  } catch (...) {
    join();
    throw;
  }
  check(join(), "join");
}

std::vector<std::unique_ptr<Data>> Engine::multiply_relinearize_rescale_batch(
    const std::vector<const Data *> &a, const std::vector<const Data *> &b, const Data &rk) {
  const std::string fn = "Multiply Relinearize Rescale Batch";
  if (a.size() != b.size() || a.empty())
    throw std::invalid_argument(fn + ": the batch lists should have one entry each per item.");
  for (size_t i = 0; i < a.size(); i++)
    if (!a[i] || !b[i]) throw std::invalid_argument(fn + ": a batch entry is null.");
  std::vector<std::unique_ptr<Data>> out(a.size());
  run_concurrent(static_cast<int>(a.size()),
                 [&](int i) { out[i] = multiply_relinearize_rescale(*a[i], *b[i], rk); });
  return out;
}

std::vector<std::unique_ptr<Data>> Engine::bootstrap_batch(const std::vector<const Data *> &cts,
                                                           const Data &rk, const Data &ck,
                                                           const BootstrapKey &bk) {
  if (cts.empty()) throw std::invalid_argument("Bootstrap Batch: the batch is empty.");
  for (const Data *c : cts)
    if (!c) throw std::invalid_argument("Bootstrap Batch: a batch entry is null.");
  std::vector<std::unique_ptr<Data>> out(cts.size());
  run_concurrent(static_cast<int>(cts.size()), [&](int i) { out[i] = bootstrap(*cts[i], rk, ck, bk); });
  return out;
}

std::vector<std::unique_ptr<Data>> Engine::multiply_rotate_batch(
    const std::vector<const Data *> &a, const std::vector<const Data *> &b, const Data &rk,
    const std::vector<const Data *> &rotation_keys) {
  const std::string fn = "Multiply Rotate Batch";
  if (a.size() != b.size() || a.size() != rotation_keys.size() || a.empty())
    throw std::invalid_argument(fn + ": the batch lists should have one entry each per item.");
  std::vector<uint64_t> key{kGraphMultiplyRotate, rk.serial};
  std::vector<const Data *> inputs;
  for (size_t i = 0; i < a.size(); i++) {
    if (!a[i] || !b[i] || !rotation_keys[i])
      throw std::invalid_argument(fn + ": a batch entry is null.");
    key.push_back(rotation_keys[i]->serial);
    inputs.push_back(a[i]);
    inputs.push_back(b[i]);
  }
  key.push_back(static_cast<uint64_t>(concurrency_));
  return run_captured(std::move(key), inputs, [&](const std::vector<const Data *> &in) {
    std::vector<std::unique_ptr<Data>> out(rotation_keys.size());
    run_concurrent(static_cast<int>(rotation_keys.size()), [&](int i) {
      auto product = multiply_relinearize_rescale(*in[2 * i], *in[2 * i + 1], rk);
      out[i] = rotate(*product, *rotation_keys[i]);
    });
    return out;
  });
}

}  // namespace fhe_b200
