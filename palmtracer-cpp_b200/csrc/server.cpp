// Serving: stacks submitted asynchronously are localized concurrently on one device.
//
// The server owns `slots` worker threads, each with its own Engine (its own CUDA stream, chunk workspace and staging
// buffers) and an equal share of the server's device-memory budget. A submitted stack waits in a FIFO queue until a
// slot is free and its estimated device memory fits in what the running stacks leave of the budget (first fit in
// submission order, so a small stack can start while a large one waits for memory). Stacks on different slots run
// on different streams, so their kernels overlap on the GPU; within a slot a stack is processed in chunks as by
// Localization. Each request records its submission, start and completion times (steady clock) for latency
// statistics. Input and output buffers stay owned by the caller and must remain valid until the request completes.
//
// Fused fits (modes 6-8): the slots' engines do not launch their own maximum-likelihood fits. Each chunk's
// candidates go to one FitBatcher, which gathers the chunks that are ready at the same time (across slots, so across
// requests) with the same fit configuration into one device work queue and fits them with ONE persistent fit launch
// on its own stream; the rows go back to each chunk's buffer and the chunk's stream continues after that launch.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace ptb {

bool LaunchFusedMle(const FitJob* jobs, int n, int lanes, Cand* fusedCands, double* fusedRows, uint32_t* offsets,
                    unsigned int* counters, cudaStream_t st);

namespace {

using Clock = std::chrono::steady_clock;

// Two jobs can share a launch when every fit setting the kernels read is the same (the spline modes: also the same
// device table).
bool SameFit(const FitParams& a, const FitParams& b)
{
	const MleParams &x = a.mle, &y = b.mle;
	bool same = a.mode == b.mode && a.roi == b.roi && x.model == y.model && x.roi == y.roi && x.maxIter == y.maxIter &&
	            x.sigma0 == y.sigma0 && x.offset == y.offset && x.gain == y.gain && x.crlbMax == y.crlbMax &&
	            x.pixelSize == y.pixelSize && x.zMin == y.zMin && x.zMax == y.zMax && x.sx == y.sx && x.sy == y.sy &&
	            x.sz == y.sz && x.dz == y.dz && x.table == y.table && x.table64 == y.table64 && a.lanes == b.lanes;
	for (int i = 0; i < 10; ++i) { same = same && x.astig[i] == y.astig[i]; }
	return same;
}

// The server's fused fit stage. Slot threads call Fit() with a chunk whose candidates are ready on the chunk's
// stream; the batcher thread waits a short window for other slots' chunks, launches one fused fit for the jobs
// with the first job's configuration (at most kMaxFitImages), and releases each caller with an event that the
// caller's stream then waits for.
class FitBatcher {
public:
	FitBatcher(int device, std::function<int()> busySlots) : device_(device), busySlots_(std::move(busySlots))
	{
		const char* w = std::getenv("PTB_FUSE_WINDOW_US");
		window_ = std::chrono::microseconds(w ? std::max(0, std::atoi(w)) : 300);
		thread_ = std::thread([this] { Loop(); });
	}

	~FitBatcher()
	{
		{
			std::lock_guard<std::mutex> g(mu_);
			stop_ = true;
		}
		cv_.notify_all();
		thread_.join();
		if (cands_) { cudaFree(cands_); }
		if (rows_) { cudaFree(rows_); }
		if (small_) { cudaFree(small_); }
		if (stream_) { cudaStreamDestroy(stream_); }
	}

	bool Fit(const FitJob& job)
	{
		Pending p;
		p.job = job;
		if (!PTB_CUDA(cudaEventCreateWithFlags(&p.ready, cudaEventDisableTiming)) ||
		    !PTB_CUDA(cudaEventCreateWithFlags(&p.done, cudaEventDisableTiming)) || !PTB_CUDA(cudaEventRecord(p.ready, job.stream))) {
			return false;
		}
		{
			std::lock_guard<std::mutex> g(mu_);
			pending_.push_back(&p);
		}
		cv_.notify_all();
		{
			std::unique_lock<std::mutex> lk(mu_);
			finished_.wait(lk, [&] { return p.finished; });
		}
		bool ok = p.ok;
		if (!ok) { SetError(p.error.empty() ? "fused fit failed" : p.error); }
		ok = ok && PTB_CUDA(cudaStreamWaitEvent(job.stream, p.done, 0));
		cudaEventDestroy(p.ready);
		cudaEventDestroy(p.done);
		return ok;
	}

	// [fused launches, chunks fitted by them]
	void Stats(uint64_t* out) const
	{
		out[0] = launches_.load();
		out[1] = jobs_.load();
	}

private:
	struct Pending {
		FitJob job;
		cudaEvent_t ready = nullptr, done = nullptr;
		bool finished = false, ok = false;
		std::string error;
	};

	void Loop()
	{
		cudaSetDevice(device_);
		const bool streamOk = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) == cudaSuccess;
		for (;;) {
			std::vector<Pending*> batch;
			{
				std::unique_lock<std::mutex> lk(mu_);
				cv_.wait(lk, [&] { return stop_ || !pending_.empty(); });
				if (pending_.empty()) { return; }  // stopping, nothing left
				// a short window for the chunks of the other busy slots
				const auto until = Clock::now() + window_;
				cv_.wait_until(lk, until, [&] { return stop_ || static_cast<int>(pending_.size()) >= busySlots_(); });
				const FitParams& key = pending_.front()->job.fp;
				for (auto it = pending_.begin(); it != pending_.end() && static_cast<int>(batch.size()) < kMaxFitImages;) {
					if (SameFit((*it)->job.fp, key)) {
						batch.push_back(*it);
						it = pending_.erase(it);
					}
					else { ++it; }
				}
			}
			ClearError();
			const bool ok = streamOk && Run(batch);
			{
				std::lock_guard<std::mutex> g(mu_);
				for (Pending* p : batch) {
					p->ok = ok;
					p->error = LastError();
					p->finished = true;
				}
			}
			finished_.notify_all();
		}
	}

	bool Run(const std::vector<Pending*>& batch)
	{
		const int n = static_cast<int>(batch.size());
		std::vector<FitJob> jobs;
		uint64_t cap = 0;
		for (Pending* p : batch) {
			jobs.push_back(p->job);
			cap += p->job.cap;
			if (!PTB_CUDA(cudaStreamWaitEvent(stream_, p->ready, 0))) { return false; }
		}
		if (cap > capacity_) {
			// the previous buffers may still be read by the last launch: free them after it
			if (!PTB_CUDA(cudaStreamSynchronize(stream_))) { return false; }
			if (cands_) { cudaFree(cands_); cands_ = nullptr; }
			if (rows_) { cudaFree(rows_); rows_ = nullptr; }
			capacity_ = 0;
			if (!PTB_CUDA(cudaMalloc(&cands_, cap * sizeof(Cand))) || !PTB_CUDA(cudaMalloc(&rows_, cap * kCols * sizeof(double)))) {
				return false;
			}
			capacity_ = cap;
		}
		if (!small_ && !PTB_CUDA(cudaMalloc(&small_, (kMaxFitImages + 1 + 3) * sizeof(uint32_t)))) { return false; }
		uint32_t* offsets = static_cast<uint32_t*>(small_);
		unsigned int* counters = static_cast<unsigned int*>(small_) + kMaxFitImages + 1;
		// the mapping the engine's Fitting export picks for the same number of points: a warp per ROI while they fill
		// the GPU a few times at most, else a thread per ROI (PTB_MLE_LANES overrides, as for every fit)
		int lanes = jobs[0].fp.lanes;
		if (lanes == 0) { lanes = cap <= 148ull * 64 ? 32 : 1; }
		if (!LaunchFusedMle(jobs.data(), n, lanes, static_cast<Cand*>(cands_), static_cast<double*>(rows_), offsets, counters,
		                    stream_)) {
			return false;
		}
		for (Pending* p : batch) {
			if (!PTB_CUDA(cudaEventRecord(p->done, stream_))) { return false; }
		}
		launches_.fetch_add(1);
		jobs_.fetch_add(static_cast<uint64_t>(n));
		return true;
	}

	int device_;
	std::function<int()> busySlots_;
	std::chrono::microseconds window_{300};
	std::mutex mu_;
	std::condition_variable cv_, finished_;
	std::deque<Pending*> pending_;
	bool stop_ = false;
	std::thread thread_;
	cudaStream_t stream_ = nullptr;
	void* cands_ = nullptr;
	void* rows_ = nullptr;
	void* small_ = nullptr;
	uint64_t capacity_ = 0;
	std::atomic<uint64_t> launches_{0}, jobs_{0};
};

struct Request {
	uint64_t id = 0;
	const uint16_t* input = nullptr;
	double* output = nullptr;
	uint64_t outputSize = 0, height = 0, width = 0, planes = 0, fit = 0;
	double thr = 0, ratio = 0;
	std::vector<double> params;
	size_t bytes = 0;
	int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
	long long written = 0;
	std::string error;
	Clock::time_point tSubmit, tStart, tDone;
};

class Server {
public:
	// Runs with `device` current: the engines (streams, pinned buffers) are created here, before any worker starts.
	Server(int device, int slots, size_t budget) : device_(device), budget_(budget)
	{
		const size_t share = budget / static_cast<size_t>(slots);
		const char* fuse = std::getenv("PTB_FUSE_FITS");
		if (!fuse || std::atoi(fuse) != 0) {
			batcher_ = std::make_unique<FitBatcher>(device, [this] { return busy_.load(); });
		}
		for (int i = 0; i < slots; ++i) {
			engines_.push_back(std::make_unique<Engine>());
			engines_.back()->SetBudget(share);
			if (batcher_) {
				FitBatcher* b = batcher_.get();
				engines_.back()->SetFitHook([b](const FitJob& job) { return b->Fit(job); });
			}
			ok_ = ok_ && engines_.back()->Init();
		}
		if (!ok_) { return; }
		for (int i = 0; i < slots; ++i) { workers_.emplace_back([this, i] { Work(i); }); }
	}

	bool Ok() const { return ok_; }

	// Stops after the running stacks; queued ones fail with "server stopped".
	~Server()
	{
		{
			std::lock_guard<std::mutex> g(mu_);
			stop_ = true;
			for (auto& r : queue_) {
				r->state = 3;
				r->error = "server stopped";
			}
			queue_.clear();
		}
		cv_.notify_all();
		done_.notify_all();
		for (auto& t : workers_) { t.join(); }
		engines_.clear();
		batcher_.reset();
	}

	void FuseStats(uint64_t* out) const
	{
		out[0] = out[1] = 0;
		if (batcher_) { batcher_->Stats(out); }
	}

	uint64_t Submit(std::shared_ptr<Request> r)
	{
		// every slot has the same budget, so engine 0's estimate holds for all (EstimateBytes only reads settings)
		r->bytes = engines_[0]->EstimateBytes(r->height, r->width, r->planes, r->outputSize);
		std::lock_guard<std::mutex> g(mu_);
		r->id = ++lastId_;
		r->tSubmit = Clock::now();
		requests_[r->id] = r;
		queue_.push_back(r);
		cv_.notify_all();
		return r->id;
	}

	// 0 queued or running, 1 done, -1 failed or unknown
	int Poll(uint64_t id)
	{
		std::lock_guard<std::mutex> g(mu_);
		auto it = requests_.find(id);
		if (it == requests_.end()) { return -1; }
		return it->second->state == 2 ? 1 : (it->second->state == 3 ? -1 : 0);
	}

	// Waits for the request, releases it and returns its doubles written (-1 on failure, message in *error).
	long long Result(uint64_t id, double* times, std::string* error)
	{
		std::unique_lock<std::mutex> lk(mu_);
		auto it = requests_.find(id);
		if (it == requests_.end()) {
			*error = "unknown request id";
			return -1;
		}
		std::shared_ptr<Request> r = it->second;
		done_.wait(lk, [&] { return r->state >= 2; });
		requests_.erase(id);
		if (times) {
			const auto sec = [&](Clock::time_point t) { return std::chrono::duration<double>(t - r->tSubmit).count(); };
			times[0] = sec(r->tStart);  // queueing delay
			times[1] = sec(r->tDone);   // latency (submission to completion)
		}
		if (r->state == 3) {
			*error = r->error;
			return -1;
		}
		return r->written;
	}

private:
	void Work(int slot)
	{
		cudaSetDevice(device_);
		Engine& engine = *engines_[slot];
		for (;;) {
			std::shared_ptr<Request> r;
			{
				std::unique_lock<std::mutex> lk(mu_);
				cv_.wait(lk, [&] { return stop_ || Admissible() != queue_.end(); });
				if (stop_) { return; }
				auto it = Admissible();
				r = *it;
				queue_.erase(it);
				inUse_ += r->bytes;
				r->state = 1;
				r->tStart = Clock::now();
				++busy_;
			}
			ClearError();
			// the device's settings (segmentation mode, fit precision) as the C ABI's calls see them
			const EngineSettings& set = SettingsFor();
			engine.SetStrict(set.strict.load());
			engine.SetPrecision(set.precision.load());
			long long n = -1;
			try {
				n = engine.Localize(r->input, false, r->output, false, r->outputSize, r->height, r->width, r->planes, r->thr,
				                    r->ratio, r->fit, r->params.empty() ? nullptr : r->params.data());
			}
			catch (const std::exception& ex) {
				SetError(ex.what());
			}
			{
				std::lock_guard<std::mutex> g(mu_);
				--busy_;
				inUse_ -= r->bytes;
				r->tDone = Clock::now();
				if (n < 0) {
					r->state = 3;
					r->error = LastError().empty() ? "localization failed" : LastError();
				}
				else {
					r->state = 2;
					r->written = n;
				}
			}
			done_.notify_all();
			cv_.notify_all();  // memory was freed: a waiting stack may now fit
		}
	}

	// First queued request whose memory fits (a stack larger than the whole budget runs alone).
	std::deque<std::shared_ptr<Request>>::iterator Admissible()
	{
		for (auto it = queue_.begin(); it != queue_.end(); ++it) {
			if (inUse_ + (*it)->bytes <= budget_ || inUse_ == 0) { return it; }
		}
		return queue_.end();
	}

	int device_;
	size_t budget_;
	size_t inUse_ = 0;
	bool stop_ = false;
	bool ok_ = true;
	uint64_t lastId_ = 0;
	std::mutex mu_;
	std::condition_variable cv_, done_;
	std::deque<std::shared_ptr<Request>> queue_;
	std::unordered_map<uint64_t, std::shared_ptr<Request>> requests_;
	std::atomic<int> busy_{0};                // slots running a stack
	std::unique_ptr<FitBatcher> batcher_;     // created before and destroyed after the engines that call it
	std::vector<std::unique_ptr<Engine>> engines_;
	std::vector<std::thread> workers_;
};

std::mutex g_serverMu;
std::unique_ptr<Server> g_server;

}  // namespace

bool ServerStart(int slots, uint64_t budgetBytes)
{
	std::lock_guard<std::mutex> g(g_serverMu);
	if (g_server) {
		SetError("server already started");
		return false;
	}
	if (slots < 1 || slots > 64) {
		SetError("server slots must be 1-64");
		return false;
	}
	int dev = 0;
	if (!PTB_CUDA(cudaGetDevice(&dev))) { return false; }
	if (budgetBytes == 0) {
		size_t freeB = 0, totalB = 0;
		if (!PTB_CUDA(cudaMemGetInfo(&freeB, &totalB))) { return false; }
		budgetBytes = freeB / 2;
	}
	g_server = std::make_unique<Server>(dev, slots, static_cast<size_t>(budgetBytes));
	if (!g_server->Ok()) {
		g_server.reset();
		return false;
	}
	return true;
}

void ServerStop()
{
	std::lock_guard<std::mutex> g(g_serverMu);
	g_server.reset();
}

uint64_t SubmitStack(const uint16_t* input, double* output, uint64_t outputSize, uint64_t height, uint64_t width, uint64_t planes,
                     double thr, double ratio, uint64_t fit, const double* fitParams, size_t nParams)
{
	std::lock_guard<std::mutex> g(g_serverMu);
	if (!g_server) {
		SetError("server not started (PTB_ServerStart)");
		return 0;
	}
	auto r = std::make_shared<Request>();
	r->input = input;
	r->output = output;
	r->outputSize = outputSize;
	r->height = height;
	r->width = width;
	r->planes = planes;
	r->thr = thr;
	r->ratio = ratio;
	r->fit = fit;
	if (fitParams && nParams) { r->params.assign(fitParams, fitParams + nParams); }
	return g_server->Submit(r);
}

int PollStack(uint64_t id)
{
	Server* s = nullptr;
	{
		std::lock_guard<std::mutex> g(g_serverMu);
		s = g_server.get();
	}
	return s ? s->Poll(id) : -1;
}

void ServerFuseStats(uint64_t* out, int n)
{
	uint64_t v[2] = {0, 0};
	{
		std::lock_guard<std::mutex> g(g_serverMu);
		if (g_server) { g_server->FuseStats(v); }
	}
	for (int k = 0; k < 2 && k < n; ++k) {
		if (out) { out[k] = v[k]; }
	}
}

long long StackResult(uint64_t id, double* times)
{
	Server* s = nullptr;
	{
		std::lock_guard<std::mutex> g(g_serverMu);
		s = g_server.get();
	}
	if (!s) {
		SetError("server not started (PTB_ServerStart)");
		return -1;
	}
	std::string err;
	const long long n = s->Result(id, times, &err);
	if (n < 0) { SetError(err); }
	return n;
}

}  // namespace ptb
