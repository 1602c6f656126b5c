// Serving loop of the C ABI (fxb_server_*): correlation jobs of different
// shapes taken as they arrive, admitted against an HBM budget, their subints
// interleaved on the device so that jobs overlap, completion detected with
// CUDA events, latency recorded per job.
//
// Three threads share the device, so that no job's host-side work holds up
// another job's kernels:
//   admitter   takes queued jobs in arrival order while the next one's device
//              footprint (fxb_job_footprint) fits the budget and fewer than
//              max_active jobs are admitted; creates the context and sets the
//              delay models;
//   submitter  round-robin over the running jobs, queues the next subint of
//              each whose next slot is free (it never waits on a busy slot
//              while another job could use the GPU); after a job's last
//              subint records an event and hands the job on;
//   reaper     once a job's event has completed reads the core result into
//              the request's buffer, marks the job done (its latency ends
//              here), then frees the context and returns its footprint.
// The CUDA context is initialised by the threads before fxb_server_create
// returns, so that no job pays for it.  Contexts take their device memory
// from the server's own memory pool, grown to the budget at creation and kept
// mapped (release threshold = budget): admitting and releasing a job then
// makes no allocation call into the driver, whose allocation and free paths
// can stall every thread of the process for tens to hundreds of
// milliseconds while other work is in flight.  Client calls (submit, poll, wait,
// stats) only touch the queue and the job table under the server's mutex.

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

#include "fxb_internal.h"

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
	bool failed = false;               // a submit failed; released without a result
	int64_t corelen = 0;
	double data_seconds = 0.0;
	// submitted, admitted, context ready, last subint submitted, completion
	// seen, result read
	clk::time_point t_submit, t_admit, t_start, t_lastsub, t_seen, t_done;
	std::string err;
};

// a thread with nothing to do polls its jobs' events this often
constexpr auto kPoll = std::chrono::microseconds(50);

}  // namespace

struct fxb_server {
	int device = 0;
	cudaMemPool_t pool = nullptr;
	size_t budget = 0, used = 0;
	int max_active = 1;
	int admitted = 0;                  // admitted and not yet released
	std::mutex mu;
	std::condition_variable cv_admit, cv_run, cv_reap, cv_done;
	std::deque<uint64_t> queue;        // waiting for admission
	std::map<uint64_t, Job> jobs;      // std::map: a Job stays put while others are added
	std::vector<uint64_t> running;     // subints still to submit
	std::vector<uint64_t> draining;    // all subints submitted, or failed
	uint64_t next_id = 1;
	bool stop = false, admitter_done = false, submitter_done = false;
	int ready = 0;                     // threads whose CUDA context is up
	cudaError_t init_err = cudaSuccess;
	std::thread admitter, submitter, reaper;
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

// bind the thread to the server's device and bring the context up
void thread_init(fxb_server *srv)
{
	cudaError_t e = cudaSetDevice(srv->device);
	if(e == cudaSuccess)
		e = cudaFree(nullptr);
	std::lock_guard<std::mutex> lk(srv->mu);
	if(e != cudaSuccess && srv->init_err == cudaSuccess)
		srv->init_err = e;
	srv->ready++;
	srv->cv_done.notify_all();
}

// context and delay models of an admitted job (no lock held)
bool start_job(fxb_server *srv, Job &j)
{
	fxb_status st = FXB_OK;
	j.ctx = fxb::create_ctx(j.req.desc, srv->pool, &st);
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

// return a released job's footprint and slot to the admitter (lock held)
void give_back(fxb_server *srv, Job &j)
{
	srv->used -= j.footprint;
	srv->admitted--;
	srv->cv_admit.notify_all();
}

void admitter_main(fxb_server *srv)
{
	thread_init(srv);
	std::unique_lock<std::mutex> lk(srv->mu);
	for(;;)
	{
		srv->cv_admit.wait(lk, [srv] {
			if(srv->stop || srv->queue.empty() || srv->admitted >= srv->max_active)
				return srv->stop;
			const Job &j = srv->jobs[srv->queue.front()];
			return srv->used + j.footprint <= srv->budget || srv->admitted == 0;   // a lone job always fits
		});
		if(srv->stop)
			break;
		Job &j = srv->jobs[srv->queue.front()];
		srv->queue.pop_front();
		srv->used += j.footprint;
		srv->admitted++;
		j.t_admit = clk::now();
		lk.unlock();
		const bool ok = start_job(srv, j);
		lk.lock();
		j.t_start = clk::now();
		if(ok)
		{
			j.state = 1;
			srv->running.push_back(j.id);
			srv->cv_run.notify_all();
		}
		else
		{
			lk.unlock();
			release_job(j);
			lk.lock();
			j.state = 3;
			srv->err = j.err;
			give_back(srv, j);
			srv->cv_done.notify_all();
		}
	}
	// stopping: fail what is still queued
	for(uint64_t id : srv->queue)
	{
		srv->jobs[id].state = 3;
		srv->jobs[id].err = "server stopped";
	}
	srv->queue.clear();
	srv->admitter_done = true;
	srv->cv_run.notify_all();
	srv->cv_done.notify_all();
}

void submitter_main(fxb_server *srv)
{
	thread_init(srv);
	std::vector<Job *> act;
	for(;;)
	{
		{
			std::unique_lock<std::mutex> lk(srv->mu);
			srv->cv_run.wait(lk, [srv] { return !srv->running.empty() || srv->admitter_done; });
			if(srv->running.empty())
				break;                         // stopping, and the admitter has handed on its last job
			act.clear();
			for(uint64_t id : srv->running)
				act.push_back(&srv->jobs[id]);
		}
		bool worked = false;
		for(Job *j : act)
		{
			if(!fxb::ctx_slot_free(j->ctx))
				continue;
			const fxb_job_request &r = j->req;
			const int S = r.desc->nstation, i = j->next_subint;
			const fxb_status st = fxb_submit_subint(j->ctx, r.bufs + (size_t)i * S, r.nbytes + (size_t)i * S,
			                                        r.datasec + (size_t)i * S, r.datans + (size_t)i * S, nullptr,
			                                        r.subsec[i], r.subns[i]);
			worked = true;
			bool finished = false;
			if(st != FXB_OK)
			{
				j->err = std::string("fxb_submit_subint: ") + fxb_last_error(j->ctx);
				j->failed = true;
				finished = true;
			}
			else if(++j->next_subint == r.nsubint)
			{
				void *stream = nullptr;
				fxb_get_stream(j->ctx, &stream);
				if(cudaEventRecord(j->done_ev, (cudaStream_t)stream) != cudaSuccess)
				{
					j->err = "cudaEventRecord failed";
					j->failed = true;
				}
				j->t_lastsub = clk::now();
				finished = true;
			}
			if(finished)
			{
				std::lock_guard<std::mutex> lk(srv->mu);
				srv->running.erase(std::find(srv->running.begin(), srv->running.end(), j->id));
				srv->draining.push_back(j->id);
				srv->cv_reap.notify_all();
			}
		}
		if(!worked)
		{
			std::unique_lock<std::mutex> lk(srv->mu);
			srv->cv_run.wait_for(lk, kPoll);
		}
	}
	std::lock_guard<std::mutex> lk(srv->mu);
	srv->submitter_done = true;
	srv->cv_reap.notify_all();
}

void reaper_main(fxb_server *srv)
{
	thread_init(srv);
	std::vector<Job *> act;
	for(;;)
	{
		{
			std::unique_lock<std::mutex> lk(srv->mu);
			srv->cv_reap.wait(lk, [srv] { return !srv->draining.empty() || srv->submitter_done; });
			if(srv->draining.empty())
				break;
			act.clear();
			for(uint64_t id : srv->draining)
				act.push_back(&srv->jobs[id]);
		}
		bool worked = false;
		for(Job *j : act)
		{
			// a failed job is released at once (fxb_destroy waits for its
			// streams, so no copy still reads the request's buffers when the
			// client learns of the failure)
			if(!j->failed && cudaEventQuery(j->done_ev) == cudaErrorNotReady)
				continue;
			worked = true;
			j->t_seen = clk::now();
			bool ok = !j->failed;
			if(ok && fxb_read_results(j->ctx, j->req.coreresult, (size_t)(2 * j->corelen)) != FXB_OK)
			{
				j->err = std::string("fxb_read_results: ") + fxb_last_error(j->ctx);
				ok = false;
			}
			if(ok)
			{
				std::lock_guard<std::mutex> lk(srv->mu);
				j->t_done = clk::now();
				j->state = 2;
				srv->latencies_ms.push_back(ms_between(j->t_submit, j->t_done));
				srv->data_seconds += j->data_seconds;
				srv->t_last = j->t_done;
				srv->draining.erase(std::find(srv->draining.begin(), srv->draining.end(), j->id));
				srv->cv_done.notify_all();
			}
			release_job(*j);
			std::lock_guard<std::mutex> lk(srv->mu);
			if(!ok)
			{
				j->t_done = clk::now();
				j->state = 3;
				srv->err = j->err;
				srv->draining.erase(std::find(srv->draining.begin(), srv->draining.end(), j->id));
				srv->cv_done.notify_all();
			}
			give_back(srv, *j);
		}
		if(!worked)
		{
			std::unique_lock<std::mutex> lk(srv->mu);
			srv->cv_reap.wait_for(lk, kPoll);
		}
	}
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

void stop_and_join(fxb_server *srv)
{
	{
		std::lock_guard<std::mutex> lk(srv->mu);
		srv->stop = true;
		srv->cv_admit.notify_all();
	}
	for(std::thread *t : {&srv->admitter, &srv->submitter, &srv->reaper})
		if(t->joinable())
			t->join();
	if(srv->pool)
		cudaMemPoolDestroy(srv->pool);
	srv->pool = nullptr;
}

// the server's pool on its device, holding up to the budget once grown, and
// grown now by one allocation of the budget (or of what the device has free,
// less a margin, if that is smaller) freed again at once
cudaError_t make_pool(fxb_server *srv)
{
	cudaError_t e = cudaSetDevice(srv->device);
	if(e != cudaSuccess)
		return e;
	cudaMemPoolProps props;
	memset(&props, 0, sizeof(props));
	props.allocType = cudaMemAllocationTypePinned;
	props.handleTypes = cudaMemHandleTypeNone;
	props.location.type = cudaMemLocationTypeDevice;
	props.location.id = srv->device;
	if((e = cudaMemPoolCreate(&srv->pool, &props)) != cudaSuccess)
		return e;
	uint64_t keep = srv->budget;
	if((e = cudaMemPoolSetAttribute(srv->pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess)
		return e;
	size_t free_b = 0, total_b = 0;
	if((e = cudaMemGetInfo(&free_b, &total_b)) != cudaSuccess)
		return e;
	const size_t margin = (size_t)2 << 30;
	const size_t grow = std::min(srv->budget, free_b > margin ? free_b - margin : 0);
	if(grow == 0)
		return cudaSuccess;
	cudaStream_t s;
	if((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess)
		return e;
	void *p = nullptr;
	e = cudaMallocFromPoolAsync(&p, grow, srv->pool, s);
	if(e == cudaSuccess)
		e = cudaFreeAsync(p, s);
	const cudaError_t e2 = cudaStreamSynchronize(s);
	cudaStreamDestroy(s);
	return e != cudaSuccess ? e : e2;
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
	const cudaError_t pe = make_pool(srv);
	if(pe != cudaSuccess)
	{
		if(srv->pool)
			cudaMemPoolDestroy(srv->pool);
		delete srv;
		if(status) *status = pe == cudaErrorMemoryAllocation ? FXB_ERR_NOMEM : FXB_ERR_CUDA;
		return nullptr;
	}
	srv->admitter = std::thread(admitter_main, srv);
	srv->submitter = std::thread(submitter_main, srv);
	srv->reaper = std::thread(reaper_main, srv);
	cudaError_t e;
	{
		std::unique_lock<std::mutex> lk(srv->mu);
		srv->cv_done.wait(lk, [srv] { return srv->ready == 3; });
		e = srv->init_err;
	}
	if(e != cudaSuccess)
	{
		stop_and_join(srv);
		delete srv;
		if(status) *status = FXB_ERR_CUDA;
		return nullptr;
	}
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
	srv->cv_admit.notify_all();
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
		if(srv->cv_done.wait_until(lk, until) == std::cv_status::timeout && it->second.state < 2)
			return FXB_ERR_TIMEOUT;
	return it->second.state == 2 ? FXB_OK : FXB_ERR_DATA;
}

FXB_API fxb_status fxb_server_job_times(fxb_server *srv, uint64_t job_id, double *phase_ms)
{
	if(!srv || !phase_ms)
		return FXB_ERR_ARG;
	std::lock_guard<std::mutex> lk(srv->mu);
	auto it = srv->jobs.find(job_id);
	if(it == srv->jobs.end())
		return FXB_ERR_ARG;
	const Job &j = it->second;
	if(j.state != 2)
		return FXB_ERR_STATE;
	phase_ms[0] = ms_between(j.t_submit, j.t_admit);
	phase_ms[1] = ms_between(j.t_admit, j.t_start);
	phase_ms[2] = ms_between(j.t_start, j.t_lastsub);
	phase_ms[3] = ms_between(j.t_lastsub, j.t_seen);
	phase_ms[4] = ms_between(j.t_seen, j.t_done);
	return FXB_OK;
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
	stop_and_join(srv);
	delete srv;
}

}  // extern "C"
