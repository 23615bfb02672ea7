// output_async.cpp - the NOUTPUT block of main.cu:73-103 off the solver's
// critical path (mcg_output_step_async, mcg_output_flush in include/mcg.h).
//
// The reference's output step stops the GPU: it sums the kinetic energy with
// a blocking copy, downloads the radial sums and the fields, and encodes and
// writes the VTI file before the next step is launched.  Here the solver's
// stream only does device-side work: it refreshes the moment planes, copies
// the five field planes and the radial sums into a device staging slot and
// encodes the VTI text and sums the kinetic energy there (tens to hundreds of
// microseconds).  A second stream then copies the slot into pinned host
// memory, and a worker thread writes the files with the same writers as
// mcg_output_step, in step order, while the solver keeps stepping.  Two
// slots: a third output step waits for the oldest.
#include <condition_variable>
#include <deque>
#include <exception>
#include <mutex>
#include <string>
#include <thread>

#include "internal.hpp"

namespace mcg {

struct AsyncOutput {
    static constexpr int kSlots = 2;
    struct Job {
        int32_t step;
        int slot;
        bool vti, radial;
        StatsSnapshot stats;
    };
    mcg_handle *h = nullptr;
    cudaStream_t io = nullptr;
    char *d_text[kSlots] = {}, *h_text[kSlots] = {};
    double *d_radial[kSlots] = {}, *h_radial[kSlots] = {};
    double *d_tke[kSlots] = {}, *h_tke[kSlots] = {};
    cudaEvent_t staged[kSlots] = {}, ready[kSlots] = {};
    bool busy[kSlots] = {};
    std::deque<Job> queue;
    std::mutex m;
    std::condition_variable cv;
    bool stop = false;
    mcg_status error = MCG_OK;
    std::string error_text;
    std::thread worker;

    void run() {
        for (;;) {
            Job job;
            {
                std::unique_lock<std::mutex> lk(m);
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                if (queue.empty()) return;
                job = queue.front();
            }
            mcg_status st = MCG_OK;
            const cudaError_t e = cudaEventSynchronize(ready[job.slot]);
            if (e != cudaSuccess) st = cuda_fail(e, "asynchronous output copy");
            try {  // an exception (allocation in a writer) becomes the reported error
                if (st == MCG_OK) {
                    tke_update(h, job.step, *h_tke[job.slot]);
                    st = io_write_tke_sample_snap(h, job.step, job.stats);
                }
                if (st == MCG_OK && job.radial) st = io_write_radial_host(h, job.stats, h_radial[job.slot]);
                if (st == MCG_OK && job.vti) {
                    char name[64];
                    std::snprintf(name, sizeof(name), "/lbm_%08d.vti", int(job.step));
                    st = io_write_vti_text(h, h->vti_dir + name, h_text[job.slot]);
                }
            } catch (const std::exception &ex) {
                st = fail(MCG_ERR_IO, std::string("asynchronous output writer: ") + ex.what());
            }
            std::lock_guard<std::mutex> lk(m);
            if (st != MCG_OK && error == MCG_OK) {
                error = st;
                error_text = mcg_last_error_string();
            }
            busy[job.slot] = false;
            queue.pop_front();
            cv.notify_all();
        }
    }
};

namespace {

mcg_status create_async(mcg_handle *h) {
    auto *a = new AsyncOutput();
    a->h = h;
    const size_t T = vti_text_layout(uint64_t(h->s.g.N)).total, M = size_t(h->p.NY) * (h->p.NX / 2);
    const bool vti = h->p.write_vti_output != 0;
    cudaError_t e = cudaStreamCreateWithFlags(&a->io, cudaStreamNonBlocking);
    for (int k = 0; k < AsyncOutput::kSlots && e == cudaSuccess; ++k) {
        if (vti) e = cudaMalloc(&a->d_text[k], T);
        if (e == cudaSuccess && vti) e = cudaMallocHost(&a->h_text[k], T);
        if (e == cudaSuccess) e = cudaMalloc(&a->d_radial[k], 5 * M * sizeof(double));
        if (e == cudaSuccess) e = cudaMallocHost(&a->h_radial[k], 5 * M * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&a->d_tke[k], sizeof(double));
        if (e == cudaSuccess) e = cudaMallocHost(&a->h_tke[k], sizeof(double));
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a->staged[k], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a->ready[k], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        h->async_out = a;
        async_release(h);
        return cuda_fail(e, "asynchronous output buffers");
    }
    a->worker = std::thread([a] { a->run(); });
    h->async_out = a;
    return MCG_OK;
}

}  // namespace

mcg_status async_flush(mcg_handle *h) {
    AsyncOutput *a = h->async_out;
    if (!a) return MCG_OK;
    std::unique_lock<std::mutex> lk(a->m);
    a->cv.wait(lk, [&] { return a->queue.empty(); });
    if (a->error != MCG_OK) {
        const mcg_status s = a->error;
        a->error = MCG_OK;
        return fail(s, a->error_text);
    }
    return MCG_OK;
}

void async_release(mcg_handle *h) {
    AsyncOutput *a = h->async_out;
    if (!a) return;
    if (a->worker.joinable()) {
        {
            std::lock_guard<std::mutex> lk(a->m);
            a->stop = true;
        }
        a->cv.notify_all();
        a->worker.join();  // the worker drains the queue before it stops
    }
    for (int k = 0; k < AsyncOutput::kSlots; ++k) {
        if (a->d_text[k]) cudaFree(a->d_text[k]);
        if (a->h_text[k]) cudaFreeHost(a->h_text[k]);
        if (a->d_radial[k]) cudaFree(a->d_radial[k]);
        if (a->h_radial[k]) cudaFreeHost(a->h_radial[k]);
        if (a->d_tke[k]) cudaFree(a->d_tke[k]);
        if (a->h_tke[k]) cudaFreeHost(a->h_tke[k]);
        if (a->staged[k]) cudaEventDestroy(a->staged[k]);
        if (a->ready[k]) cudaEventDestroy(a->ready[k]);
    }
    if (a->io) cudaStreamDestroy(a->io);
    delete a;
    h->async_out = nullptr;
}

// The device-side part of one output step; the caller has refreshed the
// moment planes on the handle's stream.
mcg_status async_enqueue(mcg_handle *h, int32_t step) {
    if (!h->async_out)
        if (mcg_status s = create_async(h)) return s;
    AsyncOutput *a = h->async_out;
    int slot = -1;
    {
        std::unique_lock<std::mutex> lk(a->m);
        a->cv.wait(lk, [&] {
            for (int k = 0; k < AsyncOutput::kSlots; ++k)
                if (!a->busy[k]) return true;
            return false;
        });
        for (int k = 0; k < AsyncOutput::kSlots; ++k)
            if (!a->busy[k]) {
                slot = k;
                break;
            }
        a->busy[slot] = true;
    }
    const size_t T = vti_text_layout(uint64_t(h->s.g.N)).total, M = size_t(h->p.NY) * (h->p.NX / 2);
    AsyncOutput::Job job{step, slot, h->p.write_vti_output != 0 && a->d_text[slot],
                         h->stats_started && h->stats_samples > 0, stats_snapshot(h)};
    cudaError_t e = cudaSuccess;
    if (job.vti) {
        e = launch_vti_encode(h->s, a->d_text[slot], h->stream);
        if (e == cudaSuccess) ++h->launches;
    }
    if (e == cudaSuccess && job.radial)
        e = cudaMemcpyAsync(a->d_radial[slot], h->s.radial, 5 * M * sizeof(double), cudaMemcpyDeviceToDevice,
                            h->stream);
    if (e == cudaSuccess) {
        e = launch_tke(h->s, a->d_tke[slot], h->stream);
        if (e == cudaSuccess) ++h->launches;
    }
    if (e == cudaSuccess) e = cudaEventRecord(a->staged[slot], h->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(a->io, a->staged[slot], 0);
    if (e == cudaSuccess && job.vti)
        e = cudaMemcpyAsync(a->h_text[slot], a->d_text[slot], T, cudaMemcpyDeviceToHost, a->io);
    if (e == cudaSuccess && job.radial)
        e = cudaMemcpyAsync(a->h_radial[slot], a->d_radial[slot], 5 * M * sizeof(double), cudaMemcpyDeviceToHost,
                            a->io);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(a->h_tke[slot], a->d_tke[slot], sizeof(double), cudaMemcpyDeviceToHost, a->io);
    if (e == cudaSuccess) e = cudaEventRecord(a->ready[slot], a->io);
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> lk(a->m);
        a->busy[slot] = false;
        return cuda_fail(e, "asynchronous output step");
    }
    {
        std::lock_guard<std::mutex> lk(a->m);
        a->queue.push_back(job);
    }
    a->cv.notify_all();
    return MCG_OK;
}

}  // namespace mcg
