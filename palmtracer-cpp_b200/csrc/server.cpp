// Serving: stacks submitted asynchronously are localized concurrently on one device.
//
// The server owns `slots` worker threads, each with its own Engine (its own CUDA stream, chunk workspace and staging
// buffers) and an equal share of the server's device-memory budget. A submitted stack waits in a FIFO queue until a
// slot is free and its estimated device memory fits in what the running stacks leave of the budget (first fit in
// submission order, so a small stack can start while a large one waits for memory). Stacks on different slots run
// on different streams, so their kernels overlap on the GPU; within a slot a stack is processed in chunks as by
// Localization. Each request records its submission, start and completion times (steady clock) for latency
// statistics. Input and output buffers stay owned by the caller and must remain valid until the request completes.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace ptb {

namespace {

using Clock = std::chrono::steady_clock;

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
		for (int i = 0; i < slots; ++i) {
			engines_.push_back(std::make_unique<Engine>());
			engines_.back()->SetBudget(share);
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
			}
			ClearError();
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
