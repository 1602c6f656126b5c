// Serving loop of the C ABI (fxb_server_*): correlation jobs of different
// shapes taken as they arrive, admitted against an HBM budget, their subints
// interleaved on the device so that jobs overlap, completion detected with
// CUDA events, latency recorded per job.
//
// One worker thread owns every context.  Per pass it
//   1. admits queued jobs in arrival order while the next one's device
//      footprint (fxb_job_footprint) fits the budget and fewer than
//      max_active jobs run: creates the context on the server's device, sets
//      the delay models,
//   2. submits one subint of each running job in turn (each context has its
//      own stream, so the kernels of different jobs run concurrently),
//   3. records an event after a job's last subint and, once it has completed,
//      reads the core result into the request's buffer, frees the context and
//      returns its footprint to the budget.
// Client calls (submit, poll, wait, stats) only touch the queue and the job
// table under the server's mutex.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fxb200.h"

namespace {

using clk = std::chrono::steady_clock;

struct Job {
	uint64_t id = 0;
	fxb_job_request req{};
	size_t footprint = 0;
	int state = 0;                     // 0 queued, 1 running, 2 done, 3 failed
	fxb_ctx *ctx = nullptr;
	cudaEvent_t done_ev = nullptr;
	int next_subint = 0;
	int64_t corelen = 0;
	double data_seconds = 0.0;
	clk::time_point t_submit, t_done;
	std::string err;
};

}  // namespace

struct fxb_server {
	int device = 0;
	size_t budget = 0, used = 0;
	int max_active = 1;
	std::mutex mu;
	std::condition_variable cv;        // worker wake-up and job completion
	std::deque<uint64_t> queue;
	std::map<uint64_t, Job> jobs;
	std::vector<uint64_t> active;
	uint64_t next_id = 1;
	bool stop = false;
	std::thread worker;
	std::string err;
	std::vector<double> latencies_ms;
	double data_seconds = 0.0;
	bool have_first = false;
	clk::time_point t_first, t_last;
};

namespace {

double ms_between(clk::time_point a, clk::time_point b)
{
	return std::chrono::duration<double, std::milli>(b - a).count();
}

// context and delay models of an admitted job (worker thread, no lock held)
bool start_job(fxb_server *srv, Job &j)
{
	fxb_status st = FXB_OK;
	j.ctx = fxb_create(j.req.desc, &st);
	if(!j.ctx)
	{
		j.err = std::string("fxb_create: ") + fxb_last_error(nullptr);
		return false;
	}
	const fxb_job_request &r = j.req;
	for(int s = 0; s < r.desc->nstation; s++)
	{
		st = fxb_set_delay_poly(j.ctx, s, r.poly_npoly[s], r.poly_order[s], r.poly0_sec[s], r.poly_interval[s],
		                        r.poly_coeffs[s]);
		if(st != FXB_OK)
		{
			j.err = std::string("fxb_set_delay_poly: ") + fxb_last_error(j.ctx);
			return false;
		}
	}
	fxb_core_result_length(j.ctx, &j.corelen);
	if(cudaEventCreateWithFlags(&j.done_ev, cudaEventDisableTiming) != cudaSuccess)
	{
		j.err = "cudaEventCreate failed";
		return false;
	}
	(void)srv;
	return true;
}

void release_job(Job &j)
{
	if(j.done_ev)
		cudaEventDestroy(j.done_ev);
	j.done_ev = nullptr;
	if(j.ctx)
		fxb_destroy(j.ctx);
	j.ctx = nullptr;
}

void worker_main(fxb_server *srv)
{
	cudaSetDevice(srv->device);
	for(;;)
	{
		// ---- 1. admission (and shutdown)
		std::vector<uint64_t> admitted;
		{
			std::unique_lock<std::mutex> lk(srv->mu);
			if(srv->stop && srv->active.empty())
				break;
			while(!srv->stop && !srv->queue.empty() && (int)srv->active.size() + (int)admitted.size() < srv->max_active)
			{
				Job &j = srv->jobs[srv->queue.front()];
				if(srv->used + j.footprint > srv->budget && !(srv->active.empty() && admitted.empty()))
					break;                              // wait for memory (a lone job is always admitted)
				srv->used += j.footprint;
				admitted.push_back(j.id);
				srv->queue.pop_front();
			}
			if(admitted.empty() && srv->active.empty())
			{
				srv->cv.wait_for(lk, std::chrono::milliseconds(2));
				continue;
			}
		}
		for(uint64_t id : admitted)
		{
			Job *j;
			{
				std::lock_guard<std::mutex> lk(srv->mu);
				j = &srv->jobs[id];
			}
			const bool ok = start_job(srv, *j);
			std::lock_guard<std::mutex> lk(srv->mu);
			if(ok)
			{
				j->state = 1;
				srv->active.push_back(id);
			}
			else
			{
				release_job(*j);
				j->state = 3;
				srv->err = j->err;
				srv->used -= j->footprint;
				srv->cv.notify_all();
			}
		}
		std::vector<uint64_t> act;
		{
			std::lock_guard<std::mutex> lk(srv->mu);
			act = srv->active;
		}
		// ---- 2. one subint of each running job
		bool worked = false;
		for(uint64_t id : act)
		{
			Job *j;
			{
				std::lock_guard<std::mutex> lk(srv->mu);
				j = &srv->jobs[id];
			}
			const fxb_job_request &r = j->req;
			if(j->next_subint >= r.nsubint)
				continue;
			const int S = r.desc->nstation, i = j->next_subint;
			fxb_status st = fxb_submit_subint(j->ctx, r.bufs + (size_t)i * S, r.nbytes + (size_t)i * S,
			                                  r.datasec + (size_t)i * S, r.datans + (size_t)i * S, nullptr, r.subsec[i],
			                                  r.subns[i]);
			worked = true;
			if(st != FXB_OK)
			{
				std::lock_guard<std::mutex> lk(srv->mu);
				j->err = std::string("fxb_submit_subint: ") + fxb_last_error(j->ctx);
				j->next_subint = r.nsubint;
				j->state = 3;
				continue;
			}
			if(++j->next_subint == r.nsubint)
			{
				void *stream = nullptr;
				fxb_get_stream(j->ctx, &stream);
				cudaEventRecord(j->done_ev, (cudaStream_t)stream);
			}
		}
		// ---- 3. completions
		for(uint64_t id : act)
		{
			Job *j;
			{
				std::lock_guard<std::mutex> lk(srv->mu);
				j = &srv->jobs[id];
			}
			if(j->next_subint < j->req.nsubint)
				continue;
			if(j->state == 1 && cudaEventQuery(j->done_ev) == cudaErrorNotReady)
				continue;
			if(j->state == 1)
			{
				fxb_status st = fxb_read_results(j->ctx, j->req.coreresult, (size_t)(2 * j->corelen));
				if(st != FXB_OK)
				{
					std::lock_guard<std::mutex> lk(srv->mu);
					j->err = std::string("fxb_read_results: ") + fxb_last_error(j->ctx);
					j->state = 3;
				}
			}
			release_job(*j);
			std::lock_guard<std::mutex> lk(srv->mu);
			j->t_done = clk::now();
			if(j->state == 1)
			{
				j->state = 2;
				srv->latencies_ms.push_back(ms_between(j->t_submit, j->t_done));
				srv->data_seconds += j->data_seconds;
				srv->t_last = j->t_done;
			}
			else
				srv->err = j->err;
			srv->used -= j->footprint;
			srv->active.erase(std::find(srv->active.begin(), srv->active.end(), id));
			worked = true;
			srv->cv.notify_all();
		}
		if(!worked)
		{
			std::unique_lock<std::mutex> lk(srv->mu);
			srv->cv.wait_for(lk, std::chrono::microseconds(200));
		}
	}
	// shutdown: fail what is still queued
	std::lock_guard<std::mutex> lk(srv->mu);
	for(uint64_t id : srv->queue)
	{
		srv->jobs[id].state = 3;
		srv->jobs[id].err = "server stopped";
	}
	srv->queue.clear();
	srv->cv.notify_all();
}

double percentile(std::vector<double> v, double p)
{
	if(v.empty())
		return 0.0;
	std::sort(v.begin(), v.end());
	const double pos = p * (double)(v.size() - 1);
	const size_t lo = (size_t)pos;
	const size_t hi = std::min(lo + 1, v.size() - 1);
	return v[lo] + (pos - (double)lo) * (v[hi] - v[lo]);
}

}  // namespace

extern "C" {

FXB_API fxb_server *fxb_server_create(int32_t device, size_t hbm_budget_bytes, int32_t max_active, fxb_status *status)
{
	int ndev = 0;
	if(cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev || max_active < 1 ||
	   hbm_budget_bytes == 0)
	{
		if(status) *status = device >= 0 && max_active >= 1 && hbm_budget_bytes ? FXB_ERR_CUDA : FXB_ERR_ARG;
		return nullptr;
	}
	fxb_server *srv = new fxb_server;
	srv->device = device;
	srv->budget = hbm_budget_bytes;
	srv->max_active = max_active;
	srv->worker = std::thread(worker_main, srv);
	if(status) *status = FXB_OK;
	return srv;
}

FXB_API fxb_status fxb_server_submit(fxb_server *srv, const fxb_job_request *req, uint64_t *job_id)
{
	if(!srv || !req || !req->desc || req->nsubint < 1 || !req->bufs || !req->nbytes || !req->datasec ||
	   !req->datans || !req->subsec || !req->subns || !req->coreresult || !req->poly_npoly || !req->poly_order ||
	   !req->poly0_sec || !req->poly_interval || !req->poly_coeffs)
		return FXB_ERR_ARG;
	size_t fp = 0;
	fxb_status st = fxb_job_footprint(req->desc, &fp);
	if(st != FXB_OK)
		return st;
	Job j;
	j.req = *req;
	j.footprint = fp;
	j.data_seconds = (double)req->nsubint * (double)req->desc->subint_ns * 1e-9;
	j.t_submit = clk::now();
	std::lock_guard<std::mutex> lk(srv->mu);
	if(srv->stop)
		return FXB_ERR_STATE;
	if(fp > srv->budget)
	{
		srv->err = "job footprint exceeds the server's HBM budget";
		return FXB_ERR_NOMEM;
	}
	j.id = srv->next_id++;
	if(!srv->have_first)
	{
		srv->have_first = true;
		srv->t_first = j.t_submit;
	}
	srv->jobs[j.id] = j;
	srv->queue.push_back(j.id);
	if(job_id) *job_id = j.id;
	srv->cv.notify_all();
	return FXB_OK;
}

FXB_API fxb_status fxb_server_poll(fxb_server *srv, uint64_t job_id, int32_t *state, double *latency_ms)
{
	if(!srv)
		return FXB_ERR_ARG;
	std::lock_guard<std::mutex> lk(srv->mu);
	auto it = srv->jobs.find(job_id);
	if(it == srv->jobs.end())
		return FXB_ERR_ARG;
	if(state) *state = it->second.state;
	if(latency_ms) *latency_ms = it->second.state == 2 ? ms_between(it->second.t_submit, it->second.t_done) : 0.0;
	return FXB_OK;
}

FXB_API fxb_status fxb_server_wait(fxb_server *srv, uint64_t job_id, double timeout_s)
{
	if(!srv)
		return FXB_ERR_ARG;
	std::unique_lock<std::mutex> lk(srv->mu);
	auto it = srv->jobs.find(job_id);
	if(it == srv->jobs.end())
		return FXB_ERR_ARG;
	const auto until = clk::now() + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(timeout_s));
	while(it->second.state < 2)
		if(srv->cv.wait_until(lk, until) == std::cv_status::timeout && it->second.state < 2)
			return FXB_ERR_TIMEOUT;
	return it->second.state == 2 ? FXB_OK : FXB_ERR_DATA;
}

FXB_API fxb_status fxb_server_stats(fxb_server *srv, int32_t *ncompleted, double *p50_ms, double *p99_ms,
                                    double *data_seconds, double *wall_seconds)
{
	if(!srv)
		return FXB_ERR_ARG;
	std::lock_guard<std::mutex> lk(srv->mu);
	if(ncompleted) *ncompleted = (int32_t)srv->latencies_ms.size();
	if(p50_ms) *p50_ms = percentile(srv->latencies_ms, 0.50);
	if(p99_ms) *p99_ms = percentile(srv->latencies_ms, 0.99);
	if(data_seconds) *data_seconds = srv->data_seconds;
	if(wall_seconds) *wall_seconds = srv->latencies_ms.empty() ? 0.0 : ms_between(srv->t_first, srv->t_last) * 1e-3;
	return FXB_OK;
}

FXB_API const char *fxb_server_last_error(const fxb_server *srv) { return srv ? srv->err.c_str() : ""; }

FXB_API void fxb_server_destroy(fxb_server *srv)
{
	if(!srv)
		return;
	{
		std::lock_guard<std::mutex> lk(srv->mu);
		srv->stop = true;
		srv->cv.notify_all();
	}
	if(srv->worker.joinable())
		srv->worker.join();
	delete srv;
}

}  // extern "C"
