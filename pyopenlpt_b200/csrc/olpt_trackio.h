// Track files: rows formatted on the device, written to disk by one writer thread per
// context in posting order (trackio.cu).
#pragma once
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>

namespace olpt {

// Runs posted jobs one after another on its own thread.  A job that throws
// std::exception records the first error; wait() returns it (and clears it), post()
// rethrows a recorded error before queueing anything new.
class FileWriter {
 public:
  FileWriter() = default;
  FileWriter(const FileWriter&) = delete;
  FileWriter& operator=(const FileWriter&) = delete;
  ~FileWriter() { stop(); }
  void post(std::function<void()> job);
  // blocks until every posted job has run; the first error since the last wait ("" if none)
  std::string wait();
  void stop();

 private:
  void loop();
  std::thread th_;
  std::mutex mu_;
  std::condition_variable cv_, idle_cv_;
  std::deque<std::function<void()>> q_;
  bool busy_ = false, quit_ = false;
  std::string err_;
};

}  // namespace olpt
