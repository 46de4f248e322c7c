// jacobi::svd::io implementation (include/io.hpp): the *.mat and *.txt matrix
// stream formats of kleedaisuki/jacobi-svd-cuda (src/io.cu).
//
// *.mat: u64 rows | u64 columns | rows*columns f64, big-endian, row-major,
// records back to back (io.hpp:40-51).  Reading maps the file (mmap) and
// decodes record by record; writing appends through a shared mapping whose
// capacity doubles from 1 MiB and is truncated to the written size on close
// (src/io.cu:497-841).  Error messages follow the reference.
#include "io.hpp"

#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <bit>
#include <cctype>
#include <cerrno>
#include <cstring>
#include <iomanip>
#include <limits>
#include <locale>
#include <sstream>
#include <stdexcept>
#include <string>
#include <system_error>

namespace jacobi::svd::io
{
    namespace
    {
        constexpr std::size_t kHeaderBytes = sizeof(MatMetaData);
        constexpr std::size_t kElementBytes = sizeof(double);
        constexpr std::size_t kMinPinnedCapacity = 64U * 1024U;
        constexpr std::size_t kMinMappedCapacity = 1U << 20;

        std::size_t mul_checked(std::size_t a, std::size_t b)
        {
            if (a != 0 && b > std::numeric_limits<std::size_t>::max() / a)
                throw std::overflow_error("Size multiplication overflow.");
            return a * b;
        }

        std::size_t add_checked(std::size_t a, std::size_t b)
        {
            if (b > std::numeric_limits<std::size_t>::max() - a)
                throw std::overflow_error("Size addition overflow.");
            return a + b;
        }

        // On-disk order is big-endian ("network order").
        std::uint64_t big_endian_u64(std::uint64_t v) noexcept
        {
            if constexpr (std::endian::native == std::endian::little)
                return __builtin_bswap64(v);
            return v;
        }

        void check_layout(const Matrix &m)
        {
            if (m.values.size() != mul_checked(m.rows, m.columns))
                throw std::invalid_argument("Matrix payload size does not match rows * columns.");
        }

        bool blank(const std::string &line)
        {
            return std::all_of(line.begin(), line.end(), [](unsigned char c) { return std::isspace(c) != 0; });
        }

        std::vector<double> parse_row(const std::string &line)
        {
            std::istringstream in(line);
            in.imbue(std::locale::classic());
            std::vector<double> row;
            double x = 0.0;
            while (in >> x)
                row.push_back(x);
            if (in.fail() && !in.eof())
                throw std::invalid_argument("Invalid numeric token in text matrix row.");
            return row;
        }

        std::streamsize to_streamsize(std::size_t bytes)
        {
            if (bytes > static_cast<std::size_t>(std::numeric_limits<std::streamsize>::max()))
                throw std::overflow_error("Byte size exceeds streamsize range.");
            return static_cast<std::streamsize>(bytes);
        }

        // Read-only mapping of a whole file.
        class MappedInput final
        {
        public:
            explicit MappedInput(const std::filesystem::path &path)
            {
                fd_ = ::open(path.c_str(), O_RDONLY | O_CLOEXEC);
                if (fd_ < 0)
                    throw std::system_error(errno, std::system_category(), "open failed");
                struct stat st{};
                if (::fstat(fd_, &st) != 0)
                {
                    const int e = errno;
                    ::close(fd_);
                    throw std::system_error(e, std::system_category(), "fstat failed");
                }
                if (st.st_size < 0)
                {
                    ::close(fd_);
                    throw std::runtime_error("Negative file size is invalid.");
                }
                size_ = static_cast<std::size_t>(st.st_size);
                if (size_ > 0)
                {
                    void *p = ::mmap(nullptr, size_, PROT_READ, MAP_SHARED, fd_, 0);
                    if (p == MAP_FAILED)
                    {
                        const int e = errno;
                        ::close(fd_);
                        throw std::system_error(e, std::system_category(), "mmap failed");
                    }
                    data_ = static_cast<const std::byte *>(p);
                    ::madvise(p, size_, MADV_SEQUENTIAL);
                }
            }
            ~MappedInput()
            {
                if (data_ != nullptr)
                    ::munmap(const_cast<std::byte *>(data_), size_);
                if (fd_ >= 0)
                    ::close(fd_);
            }
            MappedInput(const MappedInput &) = delete;
            MappedInput &operator=(const MappedInput &) = delete;
            std::span<const std::byte> bytes() const noexcept { return {data_, size_}; }

        private:
            int fd_ = -1;
            const std::byte *data_ = nullptr;
            std::size_t size_ = 0;
        };

        // Append-only output through a shared mapping; capacity doubles.
        class MappedAppendOutput final
        {
        public:
            explicit MappedAppendOutput(const std::filesystem::path &path)
            {
                fd_ = ::open(path.c_str(), O_RDWR | O_CREAT | O_TRUNC | O_CLOEXEC, 0644);
                if (fd_ < 0)
                    throw std::system_error(errno, std::system_category(), "open failed");
            }
            ~MappedAppendOutput()
            {
                try
                {
                    close();
                }
                catch (...)
                {
                }
            }
            MappedAppendOutput(const MappedAppendOutput &) = delete;
            MappedAppendOutput &operator=(const MappedAppendOutput &) = delete;

            void append(std::span<const std::byte> bytes)
            {
                if (bytes.empty())
                    return;
                reserve(add_checked(size_, bytes.size()));
                std::memcpy(data_ + size_, bytes.data(), bytes.size());
                size_ += bytes.size();
            }

            void flush()
            {
                if (data_ != nullptr && size_ > 0 && ::msync(data_, size_, MS_SYNC) != 0)
                    throw std::system_error(errno, std::system_category(), "msync failed");
            }

            // Releases the mapping and the descriptor on every path; the first
            // failure (msync, ftruncate, close) is reported after that.
            void close()
            {
                if (fd_ < 0)
                    return;
                int err = 0;
                const char *what = nullptr;
                if (data_ != nullptr && size_ > 0 && ::msync(data_, size_, MS_SYNC) != 0)
                {
                    err = errno;
                    what = "msync failed";
                }
                if (data_ != nullptr)
                    ::munmap(data_, capacity_);
                data_ = nullptr;
                if (::ftruncate(fd_, static_cast<off_t>(size_)) != 0 && what == nullptr)
                {
                    err = errno;
                    what = "ftruncate failed";
                }
                if (::close(fd_) != 0 && what == nullptr)
                {
                    err = errno;
                    what = "close failed";
                }
                fd_ = -1;
                if (what != nullptr)
                    throw std::system_error(err, std::system_category(), what);
            }

        private:
            void reserve(std::size_t need)
            {
                if (need <= capacity_)
                    return;
                std::size_t cap = capacity_ == 0 ? kMinMappedCapacity : capacity_;
                while (cap < need)
                    cap = cap > std::numeric_limits<std::size_t>::max() / 2 ? need : cap * 2;
                if (::ftruncate(fd_, static_cast<off_t>(cap)) != 0)
                    throw std::system_error(errno, std::system_category(), "ftruncate failed");
                void *p = data_ == nullptr ? ::mmap(nullptr, cap, PROT_READ | PROT_WRITE, MAP_SHARED, fd_, 0)
                                           : ::mremap(data_, capacity_, cap, MREMAP_MAYMOVE);
                if (p == MAP_FAILED)
                    throw std::system_error(errno, std::system_category(), "mmap failed");
                data_ = static_cast<std::byte *>(p);
                capacity_ = cap;
            }

            int fd_ = -1;
            std::byte *data_ = nullptr;
            std::size_t size_ = 0;
            std::size_t capacity_ = 0;
        };

        void decode_payload(const std::byte *src, std::size_t count, double *dst)
        {
            for (std::size_t i = 0; i < count; ++i)
            {
                std::uint64_t w = 0;
                std::memcpy(&w, src + i * kElementBytes, kElementBytes);
                dst[i] = std::bit_cast<double>(big_endian_u64(w));
            }
        }
    } // namespace

    // ---- PinnedHostTaskBuffer -------------------------------------------------

    PinnedHostTaskBuffer::~PinnedHostTaskBuffer() { release(); }

    PinnedHostTaskBuffer::PinnedHostTaskBuffer(PinnedHostTaskBuffer &&other) noexcept { move_from(std::move(other)); }

    PinnedHostTaskBuffer &PinnedHostTaskBuffer::operator=(PinnedHostTaskBuffer &&other) noexcept
    {
        if (this != &other)
        {
            release();
            move_from(std::move(other));
        }
        return *this;
    }

    void PinnedHostTaskBuffer::reserve(std::size_t input_bytes, std::size_t workspace_bytes)
    {
        const std::size_t need = add_checked(input_bytes, workspace_bytes);
        if (need > capacity_bytes_)
        {
            std::size_t cap = capacity_bytes_ == 0 ? kMinPinnedCapacity : capacity_bytes_;
            while (cap < need)
                cap = cap > std::numeric_limits<std::size_t>::max() / 2 ? need : cap * 2;
            void *p = nullptr;
            const cudaError_t st = ::cudaMallocHost(&p, cap);
            if (st != cudaSuccess)
                throw std::runtime_error("cudaMallocHost failed: " + std::string(::cudaGetErrorString(st)));
            release();
            data_ = static_cast<std::byte *>(p);
            capacity_bytes_ = cap;
        }
        input_size_bytes_ = input_bytes;
        workspace_size_bytes_ = workspace_bytes;
    }

    std::span<std::byte> PinnedHostTaskBuffer::mutable_input_bytes() noexcept { return {data_, input_size_bytes_}; }
    std::span<const std::byte> PinnedHostTaskBuffer::input_bytes() const noexcept { return {data_, input_size_bytes_}; }
    std::span<std::byte> PinnedHostTaskBuffer::mutable_workspace_bytes() noexcept
    {
        return {data_ + input_size_bytes_, workspace_size_bytes_};
    }
    std::span<const std::byte> PinnedHostTaskBuffer::workspace_bytes() const noexcept
    {
        return {data_ + input_size_bytes_, workspace_size_bytes_};
    }
    std::size_t PinnedHostTaskBuffer::capacity_bytes() const noexcept { return capacity_bytes_; }
    std::size_t PinnedHostTaskBuffer::input_size_bytes() const noexcept { return input_size_bytes_; }
    std::size_t PinnedHostTaskBuffer::workspace_size_bytes() const noexcept { return workspace_size_bytes_; }

    void PinnedHostTaskBuffer::release() noexcept
    {
        if (data_ != nullptr)
            (void)::cudaFreeHost(data_);
        data_ = nullptr;
        capacity_bytes_ = 0;
        input_size_bytes_ = 0;
        workspace_size_bytes_ = 0;
    }

    void PinnedHostTaskBuffer::move_from(PinnedHostTaskBuffer &&o) noexcept
    {
        data_ = std::exchange(o.data_, nullptr);
        capacity_bytes_ = std::exchange(o.capacity_bytes_, 0);
        input_size_bytes_ = std::exchange(o.input_size_bytes_, 0);
        workspace_size_bytes_ = std::exchange(o.workspace_size_bytes_, 0);
    }

    // ---- MatDispatchReader ------------------------------------------------------

    MatDispatchReader::MatDispatchReader(const std::filesystem::path &path)
        : input_(path, std::ios::in | std::ios::binary)
    {
        if (!input_)
            throw std::runtime_error("Failed to open *.mat file for dispatch reading.");
    }

    bool MatDispatchReader::read_next(MatDispatchTask &task, std::size_t workspace_bytes)
    {
        MatMetaData hdr{};
        input_.read(reinterpret_cast<char *>(&hdr), to_streamsize(kHeaderBytes));
        if (input_.gcount() == 0 && input_.eof())
            return false;
        if (input_.gcount() != to_streamsize(kHeaderBytes))
            throw std::runtime_error("Truncated *.mat header while dispatch reading.");
        const std::uint64_t rows = big_endian_u64(hdr.rows), cols = big_endian_u64(hdr.columns);
        if (rows > std::numeric_limits<std::size_t>::max() || cols > std::numeric_limits<std::size_t>::max())
            throw std::overflow_error("Matrix dimensions exceed platform size_t range.");
        const std::size_t payload = mul_checked(mul_checked(rows, cols), kElementBytes);
        // A header claiming more payload than the file holds is reported as
        // truncated before any pinned memory is reserved for it (seekable
        // files; a stream that cannot tell its position is read as it comes).
        const std::streamoff here = input_.tellg();
        if (here >= 0)
        {
            input_.seekg(0, std::ios::end);
            const std::streamoff end = input_.tellg();
            input_.seekg(here);
            if (end >= here && static_cast<std::uint64_t>(end - here) < payload)
                throw std::runtime_error("Truncated *.mat payload while dispatch reading.");
        }
        task.buffer.reserve(payload, workspace_bytes);
        if (payload > 0)
        {
            auto dst = task.buffer.mutable_input_bytes();
            input_.read(reinterpret_cast<char *>(dst.data()), to_streamsize(payload));
            if (input_.gcount() != to_streamsize(payload))
                throw std::runtime_error("Truncated *.mat payload while dispatch reading.");
        }
        task.sequence_index = next_sequence_index_;
        task.rows = static_cast<std::size_t>(rows);
        task.columns = static_cast<std::size_t>(cols);
        next_sequence_index_ = add_checked(next_sequence_index_, 1);
        return true;
    }

    Matrix decode_dispatch_task_matrix(const MatDispatchTask &task)
    {
        Matrix m;
        m.rows = task.rows;
        m.columns = task.columns;
        const std::size_t count = mul_checked(m.rows, m.columns);
        const auto payload = task.buffer.input_bytes();
        if (payload.size() != mul_checked(count, kElementBytes))
            throw std::invalid_argument("Dispatch payload size does not match rows * columns.");
        m.values.resize(count);
        decode_payload(payload.data(), count, m.values.data());
        return m;
    }

    // ---- reader / writer objects --------------------------------------------------

    struct MatReader::Impl final
    {
        MappedInput file;
        std::span<const std::byte> bytes;
        std::size_t cursor = 0;
        explicit Impl(const std::filesystem::path &p) : file(p), bytes(file.bytes()) {}
    };

    struct MatWriter::Impl final
    {
        MappedAppendOutput out;
        explicit Impl(const std::filesystem::path &p) : out(p) {}
    };

    struct TxtReader::Impl final
    {
        std::ifstream in;
        explicit Impl(const std::filesystem::path &p) : in(p, std::ios::in | std::ios::binary)
        {
            if (!in)
                throw std::runtime_error("Failed to open text matrix file for reading.");
            in.imbue(std::locale::classic());
        }
    };

    struct TxtWriter::Impl final
    {
        std::ofstream out;
        bool wrote_any = false;
        explicit Impl(const std::filesystem::path &p) : out(p, std::ios::out | std::ios::binary | std::ios::trunc)
        {
            if (!out)
                throw std::runtime_error("Failed to open text matrix file for writing.");
            out.imbue(std::locale::classic());
            out << std::setprecision(std::numeric_limits<double>::max_digits10);
        }
    };

    MatReader::MatReader(const std::filesystem::path &path) : impl_(std::make_unique<Impl>(path)) {}
    MatReader::~MatReader() = default;
    MatReader::MatReader(MatReader &&) noexcept = default;
    MatReader &MatReader::operator=(MatReader &&) noexcept = default;
    MatWriter::MatWriter(const std::filesystem::path &path) : impl_(std::make_unique<Impl>(path)) {}
    MatWriter::~MatWriter() = default;
    MatWriter::MatWriter(MatWriter &&) noexcept = default;
    MatWriter &MatWriter::operator=(MatWriter &&) noexcept = default;
    TxtReader::TxtReader(const std::filesystem::path &path) : impl_(std::make_unique<Impl>(path)) {}
    TxtReader::~TxtReader() = default;
    TxtReader::TxtReader(TxtReader &&) noexcept = default;
    TxtReader &TxtReader::operator=(TxtReader &&) noexcept = default;
    TxtWriter::TxtWriter(const std::filesystem::path &path) : impl_(std::make_unique<Impl>(path)) {}
    TxtWriter::~TxtWriter() = default;
    TxtWriter::TxtWriter(TxtWriter &&) noexcept = default;
    TxtWriter &TxtWriter::operator=(TxtWriter &&) noexcept = default;

    // ---- *.mat policy -------------------------------------------------------------

    MatFilePolicy::Reader MatFilePolicy::open_reader(const std::filesystem::path &path) { return MatReader(path); }
    MatFilePolicy::Writer MatFilePolicy::open_writer(const std::filesystem::path &path) { return MatWriter(path); }

    bool MatFilePolicy::read_next(Reader &reader, Matrix &matrix)
    {
        if (reader.impl_ == nullptr)
            throw std::runtime_error("MatReader is not initialized.");
        auto &st = *reader.impl_;
        if (st.cursor == st.bytes.size())
            return false;
        if (st.bytes.size() - st.cursor < kHeaderBytes)
            throw std::runtime_error("Truncated *.mat header.");
        MatMetaData hdr{};
        std::memcpy(&hdr, st.bytes.data() + st.cursor, kHeaderBytes);
        st.cursor += kHeaderBytes;
        const std::uint64_t rows = big_endian_u64(hdr.rows), cols = big_endian_u64(hdr.columns);
        if (rows > std::numeric_limits<std::size_t>::max() || cols > std::numeric_limits<std::size_t>::max())
            throw std::overflow_error("Matrix dimensions exceed platform size_t range.");
        matrix.rows = static_cast<std::size_t>(rows);
        matrix.columns = static_cast<std::size_t>(cols);
        const std::size_t count = mul_checked(matrix.rows, matrix.columns);
        const std::size_t payload = mul_checked(count, kElementBytes);
        if (st.bytes.size() - st.cursor < payload)
            throw std::runtime_error("Truncated *.mat payload.");
        matrix.values.resize(count);
        decode_payload(st.bytes.data() + st.cursor, count, matrix.values.data());
        st.cursor += payload;
        return true;
    }

    void MatFilePolicy::write_next(Writer &writer, const Matrix &matrix)
    {
        if (writer.impl_ == nullptr)
            throw std::runtime_error("MatWriter is not initialized.");
        check_layout(matrix);
        MatMetaData hdr{big_endian_u64(static_cast<std::uint64_t>(matrix.rows)),
                        big_endian_u64(static_cast<std::uint64_t>(matrix.columns))};
        writer.impl_->out.append(std::as_bytes(std::span<const MatMetaData>(&hdr, 1)));
        constexpr std::size_t kChunk = 32U * 1024U;
        std::vector<std::uint64_t> enc(std::min(kChunk, matrix.values.size()));
        for (std::size_t done = 0; done < matrix.values.size();)
        {
            const std::size_t k = std::min(kChunk, matrix.values.size() - done);
            for (std::size_t i = 0; i < k; ++i)
                enc[i] = big_endian_u64(std::bit_cast<std::uint64_t>(matrix.values[done + i]));
            writer.impl_->out.append(std::as_bytes(std::span<const std::uint64_t>(enc.data(), k)));
            done += k;
        }
    }

    void MatFilePolicy::flush(Writer &writer)
    {
        if (writer.impl_ == nullptr)
            throw std::runtime_error("MatWriter is not initialized.");
        writer.impl_->out.flush();
    }

    std::vector<Matrix> MatFilePolicy::read(const std::filesystem::path &path)
    {
        MatInputStream s(path);
        return s.read_all();
    }

    void MatFilePolicy::write(const std::filesystem::path &path, std::span<const Matrix> matrices)
    {
        MatOutputStream s(path);
        s.write_all(matrices);
    }

    // ---- *.txt policy -------------------------------------------------------------

    TxtFilePolicy::Reader TxtFilePolicy::open_reader(const std::filesystem::path &path) { return TxtReader(path); }
    TxtFilePolicy::Writer TxtFilePolicy::open_writer(const std::filesystem::path &path) { return TxtWriter(path); }

    bool TxtFilePolicy::read_next(Reader &reader, Matrix &matrix)
    {
        if (reader.impl_ == nullptr)
            throw std::runtime_error("TxtReader is not initialized.");
        auto &in = reader.impl_->in;
        std::vector<double> values;
        std::size_t rows = 0, cols = 0;
        bool inside = false;
        std::string line;
        while (std::getline(in, line))
        {
            if (blank(line))
            {
                if (!inside)
                    continue;
                break;
            }
            std::vector<double> row = parse_row(line);
            if (row.empty())
                throw std::invalid_argument("Text matrix row cannot be empty when line is non-blank.");
            if (!inside)
            {
                inside = true;
                cols = row.size();
            }
            else if (row.size() != cols)
            {
                throw std::invalid_argument("Inconsistent column count in text matrix block.");
            }
            values.insert(values.end(), row.begin(), row.end());
            rows = add_checked(rows, 1);
        }
        if (!inside)
        {
            if (!in.eof())
                throw std::runtime_error("Failed while reading text matrix file.");
            return false;
        }
        matrix.rows = rows;
        matrix.columns = cols;
        matrix.values = std::move(values);
        return true;
    }

    void TxtFilePolicy::write_next(Writer &writer, const Matrix &matrix)
    {
        if (writer.impl_ == nullptr)
            throw std::runtime_error("TxtWriter is not initialized.");
        check_layout(matrix);
        auto &st = *writer.impl_;
        if (st.wrote_any)
            st.out << '\n';
        for (std::size_t r = 0; r < matrix.rows; ++r)
        {
            for (std::size_t c = 0; c < matrix.columns; ++c)
            {
                if (c > 0)
                    st.out << ' ';
                st.out << matrix.values[r * matrix.columns + c];
            }
            st.out << '\n';
        }
        if (!st.out)
            throw std::runtime_error("Failed while writing text matrix file.");
        st.wrote_any = true;
    }

    void TxtFilePolicy::flush(Writer &writer)
    {
        if (writer.impl_ == nullptr)
            throw std::runtime_error("TxtWriter is not initialized.");
        writer.impl_->out.flush();
        if (!writer.impl_->out)
            throw std::runtime_error("Failed to flush text matrix file.");
    }

    std::vector<Matrix> TxtFilePolicy::read(const std::filesystem::path &path)
    {
        TxtInputStream s(path);
        return s.read_all();
    }

    void TxtFilePolicy::write(const std::filesystem::path &path, std::span<const Matrix> matrices)
    {
        TxtOutputStream s(path);
        s.write_all(matrices);
    }

    std::vector<Matrix> read_mat_file(const std::filesystem::path &path) { return MatFilePolicy::read(path); }
    void write_mat_file(const std::filesystem::path &path, std::span<const Matrix> m) { MatFilePolicy::write(path, m); }
    std::vector<Matrix> read_txt_file(const std::filesystem::path &path) { return TxtFilePolicy::read(path); }
    void write_txt_file(const std::filesystem::path &path, std::span<const Matrix> m) { TxtFilePolicy::write(path, m); }
} // namespace jacobi::svd::io
