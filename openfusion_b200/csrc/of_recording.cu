// of_recording.cu -- recorded depth sequences in the reference's on-disk
// format, and a prefetching reader that feeds them to the device.
//
// Format (Source/data/ParametersFileFormat.txt:1-11, written by
// WriteToFile::~WriteToFile, Source/src/CameraSupport/WriteToFile.cpp:18-63,
// read by CameraFromFile::Init, CameraFromFile.cpp:22-70): a directory with
// `Parameters.txt` (width, height, fx fy, cx cy, z offset mm, min depth mm,
// max depth mm, number of frames, name, date, camera type; one item per
// line, numbers whitespace-separated) and one raw file per frame,
// `recorded<N>` for N = 1, 2, ...: width x height uint16 depth in mm, row
// major, native byte order (CameraFromFile::GetDepthFrame, :73-98;
// WriteToFile::GetDepthFrame, :117-145).
//
// The reader (of_reader_*) keeps a ring of pinned host buffers filled by one
// background thread, frames ahead of the caller; of_reader_next copies the
// next frame to the device with one cudaMemcpyAsync on the caller's stream
// and records an event, and a buffer is refilled only after its copy's event
// has completed.
#include "of_common.cuh"

#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

namespace {

std::string frame_path(const char *dir, int number) {
  std::string p(dir);
  if (!p.empty() && p.back() != '/') p += '/';
  return p + "recorded" + std::to_string(number);
}

std::string params_path(const char *dir) {
  std::string p(dir);
  if (!p.empty() && p.back() != '/') p += '/';
  return p + "Parameters.txt";
}

void copy_field(char *dst, size_t cap, const std::string &s) {
  const size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
  memcpy(dst, s.data(), n);
  dst[n] = 0;
}

of_status_t read_frame_file(const char *dir, int number, int w, int h, uint16_t *dst) {
  std::ifstream f(frame_path(dir, number), std::ios::binary);
  if (!f.is_open()) return OF_ERR_IO;
  const std::streamsize bytes = (std::streamsize)w * h * (std::streamsize)sizeof(uint16_t);
  f.read(reinterpret_cast<char *>(dst), bytes);
  return f.gcount() == bytes ? OF_OK : OF_ERR_IO;
}

}  // namespace

extern "C" of_status_t of_recording_read_info(const char *dir, of_recording_info_t *info) {
  if (!dir || !info) return OF_ERR_INVALID_ARGUMENT;
  std::ifstream f(params_path(dir));
  if (!f.is_open()) return OF_ERR_IO;
  memset(info, 0, sizeof(*info));
  of_camera_t &c = info->camera;
  if (!(f >> c.width >> c.height >> c.fx >> c.fy >> c.cx >> c.cy >> info->z_offset_mm >>
        c.min_depth_mm >> c.max_depth_mm))
    return OF_ERR_IO;
  if (c.width <= 0 || c.height <= 0 || c.fx <= 0.f || c.fy <= 0.f) return OF_ERR_IO;
  // the reader of the reference stops here (CameraFromFile.cpp:33-37); the
  // recorder also writes the frame count, name, date and camera type
  int frames = 0;
  if (f >> frames) info->frames = frames;
  std::string line;
  std::getline(f, line);  // rest of the frame-count line
  std::string fields[3];
  for (int i = 0; i < 3 && std::getline(f, line); ++i) {
    while (!line.empty() && (line.back() == '\r' || line.back() == ' ')) line.pop_back();
    fields[i] = line;
  }
  copy_field(info->name, sizeof(info->name), fields[0]);
  copy_field(info->date, sizeof(info->date), fields[1]);
  copy_field(info->camera_type, sizeof(info->camera_type), fields[2]);
  return OF_OK;
}

extern "C" of_status_t of_recording_write_info(const char *dir, const of_recording_info_t *info) {
  if (!dir || !info) return OF_ERR_INVALID_ARGUMENT;
  std::ofstream f(params_path(dir));
  if (!f.is_open()) return OF_ERR_IO;
  const of_camera_t &c = info->camera;
  char buf[512];
  // the recorder's line layout (WriteToFile.cpp:32-58)
  snprintf(buf, sizeof buf, "%d\n%d\n%.9g %.9g\n%.9g %.9g\n%.9g\n%.9g\n%.9g\n%d\n", c.width,
           c.height, (double)c.fx, (double)c.fy, (double)c.cx, (double)c.cy,
           (double)info->z_offset_mm, (double)c.min_depth_mm, (double)c.max_depth_mm,
           info->frames);
  f << buf << info->name << "\n" << info->date << "\n" << info->camera_type << "\n";
  f.flush();
  return f.good() ? OF_OK : OF_ERR_IO;
}

extern "C" of_status_t of_recording_read_frame(const char *dir, int32_t number, int32_t width,
                                               int32_t height, uint16_t *depth) {
  if (!dir || !depth || number < 1 || width <= 0 || height <= 0) return OF_ERR_INVALID_ARGUMENT;
  return read_frame_file(dir, number, width, height, depth);
}

extern "C" of_status_t of_recording_write_frame(const char *dir, int32_t number, int32_t width,
                                                int32_t height, const uint16_t *depth,
                                                int32_t depth_is_device, of_stream_t stream) {
  if (!dir || !depth || number < 1 || width <= 0 || height <= 0) return OF_ERR_INVALID_ARGUMENT;
  const size_t bytes = (size_t)width * height * sizeof(uint16_t);
  std::vector<uint16_t> host;
  const uint16_t *src = depth;
  if (depth_is_device) {
    host.resize((size_t)width * height);
    OF_CUDA_TRY(cudaMemcpyAsync(host.data(), depth, bytes, cudaMemcpyDeviceToHost,
                                (cudaStream_t)stream));
    OF_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    src = host.data();
  }
  std::ofstream f(frame_path(dir, number), std::ios::binary);
  if (!f.is_open()) return OF_ERR_IO;
  f.write(reinterpret_cast<const char *>(src), (std::streamsize)bytes);
  f.flush();
  return f.good() ? OF_OK : OF_ERR_IO;
}

// ------------------------------------------------------------ prefetching --

struct of_reader {
  std::string dir;
  int w = 0, h = 0, frames = 0;
  struct Slot {
    uint16_t *host = nullptr;  // pinned
    cudaEvent_t copied = nullptr;
    int number = 0;       // frame held (0 = none)
    bool ready = false;   // filled and not yet handed out
    bool in_flight = false;  // handed out: its copy may still run
    of_status_t status = OF_OK;
  };
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  bool stop = false;
  int next_fill = 1;  // next frame number the worker reads
  int next_out = 1;   // next frame number handed to the caller
};

namespace {

void reader_main(of_reader *r) {
  const int n = (int)r->slots.size();
  for (;;) {
    int number, si;
    {
      std::unique_lock<std::mutex> lk(r->mu);
      // a free slot: the one the next frame maps to, once handed out and copied
      r->cv.wait(lk, [&] {
        if (r->stop || r->next_fill > r->frames) return true;
        const of_reader::Slot &s = r->slots[(r->next_fill - 1) % n];
        return !s.ready;
      });
      if (r->stop || r->next_fill > r->frames) return;
      number = r->next_fill++;
      si = (number - 1) % n;
    }
    of_reader::Slot &s = r->slots[si];
    // the copy of the frame this slot held last must have finished
    if (s.in_flight) cudaEventSynchronize(s.copied);
    const of_status_t st = read_frame_file(r->dir.c_str(), number, r->w, r->h, s.host);
    {
      std::lock_guard<std::mutex> lk(r->mu);
      s.in_flight = false;
      s.number = number;
      s.status = st;
      s.ready = true;
    }
    r->cv.notify_all();
  }
}

void reader_free(of_reader *r) {
  if (r->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lk(r->mu);
      r->stop = true;
    }
    r->cv.notify_all();
    r->worker.join();
  }
  for (auto &s : r->slots) {
    if (s.copied) {
      cudaEventSynchronize(s.copied);
      cudaEventDestroy(s.copied);
    }
    if (s.host) cudaFreeHost(s.host);
  }
  delete r;
}

}  // namespace

extern "C" of_status_t of_reader_open(const char *dir, int32_t prefetch, of_reader_t *out) {
  if (!dir || !out || prefetch < 1 || prefetch > 64) return OF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  of_recording_info_t info;
  of_status_t st = of_recording_read_info(dir, &info);
  if (st != OF_OK) return st;
  of_reader *r = new (std::nothrow) of_reader();
  if (!r) return OF_ERR_OUT_OF_MEMORY;
  r->dir = dir;
  r->w = info.camera.width;
  r->h = info.camera.height;
  r->frames = info.frames;
  if (r->frames <= 0) {
    // no frame count: as many consecutive recorded<N> files as exist
    int n = 0;
    while (std::ifstream(frame_path(dir, n + 1), std::ios::binary).is_open()) ++n;
    r->frames = n;
  }
  r->slots.resize(prefetch);
  const size_t bytes = (size_t)r->w * r->h * sizeof(uint16_t);
  for (auto &s : r->slots) {
    cudaError_t e = cudaHostAlloc(&s.host, bytes, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      reader_free(r);
      return of_set_cuda_error(e);
    }
  }
  r->worker = std::thread(reader_main, r);
  *out = r;
  return OF_OK;
}

extern "C" of_status_t of_reader_info(of_reader_t r, int32_t *width, int32_t *height,
                                      int32_t *frames) {
  if (!r) return OF_ERR_INVALID_ARGUMENT;
  if (width) *width = r->w;
  if (height) *height = r->h;
  if (frames) *frames = r->frames;
  return OF_OK;
}

extern "C" of_status_t of_reader_next(of_reader_t r, uint16_t *d_depth, of_stream_t stream) {
  if (!r || !d_depth) return OF_ERR_INVALID_ARGUMENT;
  const int n = (int)r->slots.size();
  std::unique_lock<std::mutex> lk(r->mu);
  if (r->next_out > r->frames) return OF_END_OF_SEQUENCE;
  of_reader::Slot &s = r->slots[(r->next_out - 1) % n];
  r->cv.wait(lk, [&] { return s.ready && s.number == r->next_out; });
  if (s.status != OF_OK) return s.status;
  const size_t bytes = (size_t)r->w * r->h * sizeof(uint16_t);
  cudaError_t e = cudaMemcpyAsync(d_depth, s.host, bytes, cudaMemcpyHostToDevice,
                                  (cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaEventRecord(s.copied, (cudaStream_t)stream);
  if (e != cudaSuccess) return of_set_cuda_error(e);
  s.ready = false;
  s.in_flight = true;
  r->next_out += 1;
  lk.unlock();
  r->cv.notify_all();
  return OF_OK;
}

extern "C" of_status_t of_reader_close(of_reader_t r) {
  if (!r) return OF_ERR_INVALID_ARGUMENT;
  reader_free(r);
  return OF_OK;
}
