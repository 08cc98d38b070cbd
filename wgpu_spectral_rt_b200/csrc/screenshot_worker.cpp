// screenshot_worker.cpp — PNG encoding off the caller's thread.
//
// The reference's engine hands every screenshot to a saver thread over a
// channel (src/engine.rs:39-45 spawns it, :242 sends the read-back pixels)
// and that thread flips, sRGB-encodes and writes the PNG
// (src/screenshot.rs:27-103).  Here one library-owned worker thread, started
// by the first asynchronous write, takes jobs from a queue in order; a job
// owns a copy of its pixels, so the caller's buffer is free on return.
// srt_screenshot_flush waits until the queue is empty and reports the writes
// that failed since the previous flush.  At process exit the worker finishes
// the queued jobs before the library unloads.  A process that forks after
// its first asynchronous write has no worker in the child.
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <system_error>
#include <thread>
#include <utility>
#include <vector>

#include "host_scene.h"

namespace {

struct ScreenshotJob {
    std::string path;
    std::vector<uint8_t> rgba;
    uint32_t w, h, pitch;
};

class ScreenshotWorker {
public:
    ~ScreenshotWorker() {
        {
            std::lock_guard<std::mutex> l(m_);
            stop_ = true;
        }
        work_.notify_all();
        if (thread_.joinable()) thread_.join();
    }
    void push(ScreenshotJob&& job) {
        std::lock_guard<std::mutex> l(m_);
        if (!thread_.joinable()) thread_ = std::thread([this] { run(); });
        queue_.push_back(std::move(job));
        ++pending_;
        work_.notify_one();
    }
    uint32_t flush() {
        std::unique_lock<std::mutex> l(m_);
        idle_.wait(l, [this] { return pending_ == 0; });
        const uint32_t f = failed_;
        failed_ = 0;
        return f;
    }

private:
    void run() {
        std::unique_lock<std::mutex> l(m_);
        for (;;) {
            work_.wait(l, [this] { return stop_ || !queue_.empty(); });
            if (queue_.empty()) return;  // stopping, and every job is written
            ScreenshotJob job = std::move(queue_.front());
            queue_.pop_front();
            l.unlock();
            const bool ok = write_screenshot_png(job.path, job.rgba.data(), job.w, job.h, job.pitch);
            l.lock();
            if (!ok) ++failed_;
            if (--pending_ == 0) idle_.notify_all();
        }
    }
    std::mutex m_;
    std::condition_variable work_, idle_;
    std::deque<ScreenshotJob> queue_;
    std::thread thread_;
    size_t pending_ = 0;
    uint32_t failed_ = 0;
    bool stop_ = false;
};

ScreenshotWorker& worker() {
    static ScreenshotWorker w;
    return w;
}

}  // namespace

void screenshot_enqueue(const std::string& path, std::vector<uint8_t>&& rgba, uint32_t w, uint32_t h,
                        uint32_t pitch) {
    worker().push(ScreenshotJob{path, std::move(rgba), w, h, pitch});
}

extern "C" srt_status srt_screenshot_write_async(const char* path, const uint8_t* rgba, uint32_t w, uint32_t h,
                                                 uint32_t pitch) {
    if (!path || !rgba || w == 0 || h == 0 || pitch < 4 * w) return SRT_ERR_INVALID_ARG;
    try {
        // rows of `pitch` bytes; the last row needs only its 4 w pixel bytes
        std::vector<uint8_t> copy((size_t)pitch * h);
        std::memcpy(copy.data(), rgba, (size_t)pitch * (h - 1) + 4u * w);
        screenshot_enqueue(path, std::move(copy), w, h, pitch);
    } catch (const std::bad_alloc&) {
        return SRT_ERR_OOM;
    } catch (const std::system_error&) {  // the worker thread could not start
        return SRT_ERR_OOM;
    }
    return SRT_OK;
}

extern "C" srt_status srt_screenshot_flush(uint32_t* failed_writes) {
    const uint32_t f = worker().flush();
    if (failed_writes) *failed_writes = f;
    return SRT_OK;
}
