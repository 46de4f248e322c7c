// The io.hpp policy concepts as an extension point (built and run by
// tests/test_io.py; no GPU): the file policies satisfy the concepts, a
// policy without flush does not satisfy MatrixOutputPolicy, and a
// user-defined in-memory policy works with the stream templates.
#include <iostream>
#include <vector>

#include "io.hpp"

using namespace jacobi::svd::io;

static_assert(MatrixInputPolicy<MatFilePolicy> && MatrixOutputPolicy<MatFilePolicy>);
static_assert(MatrixInputPolicy<TxtFilePolicy> && MatrixOutputPolicy<TxtFilePolicy>);

// Three 2 x 2 matrices read from memory; everything written is kept.
struct MemoryPolicy
{
    struct Reader
    {
        int next = 0;
    };
    struct Writer
    {
        std::vector<Matrix> *sink = nullptr;
        int flushes = 0;
    };
    static std::vector<Matrix> written;
    static Reader open_reader(const std::filesystem::path &) { return Reader{}; }
    static bool read_next(Reader &r, Matrix &m)
    {
        if (r.next == 3)
            return false;
        const double k = r.next++;
        m = Matrix{2, 2, {k, k + 1, k + 2, k + 3}};
        return true;
    }
    static Writer open_writer(const std::filesystem::path &) { return Writer{&written, 0}; }
    static void write_next(Writer &w, const Matrix &m) { w.sink->push_back(m); }
    static void flush(Writer &w) { ++w.flushes; }
};
std::vector<Matrix> MemoryPolicy::written;

struct NoFlushPolicy
{
    struct Writer
    {
    };
    static Writer open_writer(const std::filesystem::path &) { return {}; }
    static void write_next(Writer &, const Matrix &) {}
};
static_assert(MatrixInputPolicy<MemoryPolicy> && MatrixOutputPolicy<MemoryPolicy>);
static_assert(!MatrixOutputPolicy<NoFlushPolicy>);

int main()
{
    MatrixInputStream<MemoryPolicy> in("unused");
    MatrixOutputStream<MemoryPolicy> out("unused");
    const std::vector<Matrix> all = in.read_all();
    out.write_all(all);
    std::cout << all.size() << ' ' << MemoryPolicy::written.size() << ' ' << in.eof();
    for (const Matrix &m : MemoryPolicy::written)
        std::cout << ' ' << m.values[0] + m.values[3];
    std::cout << '\n';
    return 0;
}
