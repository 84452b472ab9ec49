// Frame files and conservation totals from device state (the reference's
// lib/2d/Output.cpp, WriteQhelp.cpp and ConSoln.cpp), used by the solver's
// C ABI in finess_b200.cu.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <string>
#include <thread>

namespace fin {
namespace io {

// One value of a frame or conservation file as the reference's iostreams
// print it: setprecision(16), setw(24), scientific, i.e. "%24.16e".  Every
// finite or non-finite double takes at most 24 characters, so each line of
// a frame file is exactly 25 bytes.
constexpr int RECORD = 25;

// Formats n values as consecutive 25-byte lines ("%24.16e\n") into out
// (n * 25 bytes, plus one byte for the terminating NUL), on up to nthreads
// host threads.
void format_records(const double* v, size_t n, char* out, int nthreads);

// Parses n values from the text of a frame file body (after its header line):
// fast path for 25-byte lines, else whitespace-separated numbers.  Returns
// false when fewer than n numbers are found.
bool parse_records(const char* text, size_t len, double* v, size_t n, int nthreads);

// Asynchronous writer of q%04d.dat / a%04d.dat: the state's interior is
// reordered on the device into the files' order (component, then j, then i
// fastest: lib/2d/Output.cpp:39-45), copied to pinned host memory on a side
// stream (the solver's stream runs on as soon as the reorder is done), then
// formatted and written by a host thread.
class FrameWriter {
public:
    FrameWriter() = default;
    ~FrameWriter();
    FrameWriter(const FrameWriter&) = delete;
    FrameWriter& operator=(const FrameWriter&) = delete;
    // Starts writing q (ncomp planes of mx x my, plane pitch `plane`) and aux
    // (naux planes, may be 0; aux null: zeros) at time t.  Waits for the
    // previous frame first.
    // Returns 0 or a FIN_ERR_* code (message in err()).
    int start(cudaStream_t stream, const double* q, int ncomp, const double* aux, int naux, size_t plane, int mx,
              int my, double t, const std::string& qpath, const std::string& apath);
    // Waits until the last frame is on disk; its status.
    int wait();
    const std::string& err() const { return err_; }

private:
    int ensure(size_t n);
    double* d_stage_ = nullptr;   // device, [c][j][i]
    double* h_stage_ = nullptr;   // pinned host
    size_t cap_ = 0;              // doubles
    cudaStream_t side_ = nullptr;
    cudaEvent_t ready_ = nullptr, copied_ = nullptr;
    std::thread worker_;
    int status_ = 0;
    std::string err_;
};

// Writes "%24.16e " for t and each total, then a newline, to path; truncates
// the file first when t == 0 and appends otherwise (lib/2d/ConSoln.cpp:39-46,
// 87-95, totals below 1e-99 in magnitude printed as 0).
int append_conservation(const std::string& path, double t, const double* totals, int ncomp);

// Per-component totals dx*dy*sum(q) over the interior on the device, written
// to d_out[ncomp] on the stream: one CTA per (component, chunk) with
// compensated partial sums, combined in a fixed order (deterministic).
// d_scratch holds 2 * ncomp * NCHUNK doubles.
constexpr int NCHUNK = 256;
void launch_totals(cudaStream_t stream, const double* q, int ncomp, size_t plane, size_t n, double dxdy,
                   double* d_scratch, double* d_out);

// Reads a frame file (header line t, then ncomp * mx * my values in the
// files' order) and uploads it as planes into q (plane pitch `plane`) through
// d_stage (ncomp * mx * my doubles).
int read_frame(const std::string& path, cudaStream_t stream, double* q, int ncomp, size_t plane, int mx, int my,
               double* d_stage, double* t, std::string* err);

}  // namespace io
}  // namespace fin
