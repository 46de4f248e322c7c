// jacobi::svd::io - the matrix stream formats, source-compatible with
// kleedaisuki/jacobi-svd-cuda include/io.hpp (same namespace, types,
// policies, concepts, stream templates and free functions).  Implemented by
// jacobi-svd-cuda_b200/csrc/io.cpp.
//
// *.mat: records of  u64 rows | u64 columns | rows*columns f64, big-endian,
// row-major, concatenated with no file header (reference io.hpp:40-51).
// *.txt: one matrix per block of whitespace-separated rows; blocks are
// separated by blank lines; values printed with max_digits10.
#pragma once

#include <concepts>
#include <cstddef>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <memory>
#include <span>
#include <utility>
#include <vector>

namespace jacobi::svd::io
{
    /// Row-major FP64 matrix.
    struct Matrix final
    {
        std::size_t rows = 0;
        std::size_t columns = 0;
        std::vector<double> values;
    };

    /// *.mat record header; stored in network byte order on disk.
    struct MatMetaData final
    {
        std::uint64_t rows = 0;
        std::uint64_t columns = 0;
    };

    /// One pinned (cudaMallocHost) block split into an input region and a
    /// workspace region; grows by doubling from 64 KiB (reference :57-170).
    class PinnedHostTaskBuffer final
    {
    public:
        PinnedHostTaskBuffer() = default;
        ~PinnedHostTaskBuffer();
        PinnedHostTaskBuffer(const PinnedHostTaskBuffer &) = delete;
        PinnedHostTaskBuffer &operator=(const PinnedHostTaskBuffer &) = delete;
        PinnedHostTaskBuffer(PinnedHostTaskBuffer &&other) noexcept;
        PinnedHostTaskBuffer &operator=(PinnedHostTaskBuffer &&other) noexcept;

        void reserve(std::size_t input_bytes, std::size_t workspace_bytes);
        [[nodiscard]] std::span<std::byte> mutable_input_bytes() noexcept;
        [[nodiscard]] std::span<const std::byte> input_bytes() const noexcept;
        [[nodiscard]] std::span<std::byte> mutable_workspace_bytes() noexcept;
        [[nodiscard]] std::span<const std::byte> workspace_bytes() const noexcept;
        [[nodiscard]] std::size_t capacity_bytes() const noexcept;
        [[nodiscard]] std::size_t input_size_bytes() const noexcept;
        [[nodiscard]] std::size_t workspace_size_bytes() const noexcept;

    private:
        void release() noexcept;
        void move_from(PinnedHostTaskBuffer &&other) noexcept;

        std::byte *data_ = nullptr;
        std::size_t capacity_bytes_ = 0;
        std::size_t input_size_bytes_ = 0;
        std::size_t workspace_size_bytes_ = 0;
    };

    /// One *.mat record read by MatDispatchReader: raw big-endian payload in
    /// the pinned input region.
    struct MatDispatchTask final
    {
        std::size_t sequence_index = 0;
        std::size_t rows = 0;
        std::size_t columns = 0;
        PinnedHostTaskBuffer buffer;
    };

    /// Sequential *.mat reader that copies each record's raw bytes into a
    /// task's pinned buffer (reference :207-234).
    class MatDispatchReader final
    {
    public:
        explicit MatDispatchReader(const std::filesystem::path &path);
        /// Reads the next record; false at end of file.
        [[nodiscard]] bool read_next(MatDispatchTask &task, std::size_t workspace_bytes = 0);

    private:
        std::ifstream input_;
        std::size_t next_sequence_index_ = 0;
    };

    /// Decodes a dispatch task's big-endian payload into a Matrix.
    [[nodiscard]] Matrix decode_dispatch_task_matrix(const MatDispatchTask &task);

    class MatReader;
    class MatWriter;
    class TxtReader;
    class TxtWriter;

    /// *.mat policy: memory-mapped reader, append-mapped writer.
    struct MatFilePolicy final
    {
        using Reader = MatReader;
        using Writer = MatWriter;
        [[nodiscard]] static Reader open_reader(const std::filesystem::path &path);
        [[nodiscard]] static Writer open_writer(const std::filesystem::path &path);
        [[nodiscard]] static bool read_next(Reader &reader, Matrix &matrix);
        static void write_next(Writer &writer, const Matrix &matrix);
        static void flush(Writer &writer);
        [[nodiscard]] static std::vector<Matrix> read(const std::filesystem::path &path);
        static void write(const std::filesystem::path &path, std::span<const Matrix> matrices);
    };

    /// *.txt policy.
    struct TxtFilePolicy final
    {
        using Reader = TxtReader;
        using Writer = TxtWriter;
        [[nodiscard]] static Reader open_reader(const std::filesystem::path &path);
        [[nodiscard]] static Writer open_writer(const std::filesystem::path &path);
        [[nodiscard]] static bool read_next(Reader &reader, Matrix &matrix);
        static void write_next(Writer &writer, const Matrix &matrix);
        static void flush(Writer &writer);
        [[nodiscard]] static std::vector<Matrix> read(const std::filesystem::path &path);
        static void write(const std::filesystem::path &path, std::span<const Matrix> matrices);
    };

    class MatReader final
    {
    public:
        explicit MatReader(const std::filesystem::path &path);
        ~MatReader();
        MatReader(const MatReader &) = delete;
        MatReader &operator=(const MatReader &) = delete;
        MatReader(MatReader &&other) noexcept;
        MatReader &operator=(MatReader &&other) noexcept;

    private:
        struct Impl;
        std::unique_ptr<Impl> impl_;
        friend struct MatFilePolicy;
    };

    class MatWriter final
    {
    public:
        explicit MatWriter(const std::filesystem::path &path);
        ~MatWriter();
        MatWriter(const MatWriter &) = delete;
        MatWriter &operator=(const MatWriter &) = delete;
        MatWriter(MatWriter &&other) noexcept;
        MatWriter &operator=(MatWriter &&other) noexcept;

    private:
        struct Impl;
        std::unique_ptr<Impl> impl_;
        friend struct MatFilePolicy;
    };

    class TxtReader final
    {
    public:
        explicit TxtReader(const std::filesystem::path &path);
        ~TxtReader();
        TxtReader(const TxtReader &) = delete;
        TxtReader &operator=(const TxtReader &) = delete;
        TxtReader(TxtReader &&other) noexcept;
        TxtReader &operator=(TxtReader &&other) noexcept;

    private:
        struct Impl;
        std::unique_ptr<Impl> impl_;
        friend struct TxtFilePolicy;
    };

    class TxtWriter final
    {
    public:
        explicit TxtWriter(const std::filesystem::path &path);
        ~TxtWriter();
        TxtWriter(const TxtWriter &) = delete;
        TxtWriter &operator=(const TxtWriter &) = delete;
        TxtWriter(TxtWriter &&other) noexcept;
        TxtWriter &operator=(TxtWriter &&other) noexcept;

    private:
        struct Impl;
        std::unique_ptr<Impl> impl_;
        friend struct TxtFilePolicy;
    };

    /// A policy that can open a reader and pull matrices from it.
    template <typename Policy>
    concept MatrixInputPolicy = requires(const std::filesystem::path &path, typename Policy::Reader &reader,
                                         Matrix &matrix) {
        typename Policy::Reader;
        { Policy::open_reader(path) } -> std::same_as<typename Policy::Reader>;
        { Policy::read_next(reader, matrix) } -> std::same_as<bool>;
    };

    /// A policy that can open a writer, push matrices and flush.
    template <typename Policy>
    concept MatrixOutputPolicy = requires(const std::filesystem::path &path, typename Policy::Writer &writer,
                                          const Matrix &matrix) {
        typename Policy::Writer;
        { Policy::open_writer(path) } -> std::same_as<typename Policy::Writer>;
        { Policy::write_next(writer, matrix) } -> std::same_as<void>;
        { Policy::flush(writer) } -> std::same_as<void>;
    };

    /// Pull-style matrix stream over an input policy.
    template <MatrixInputPolicy Policy>
    class MatrixInputStream final
    {
    public:
        explicit MatrixInputStream(const std::filesystem::path &path) : reader_(Policy::open_reader(path)) {}

        bool read_one(Matrix &matrix)
        {
            if (eof_)
                return false;
            const bool got = Policy::read_next(reader_, matrix);
            eof_ = !got;
            return got;
        }

        MatrixInputStream &operator>>(Matrix &matrix)
        {
            (void)read_one(matrix);
            return *this;
        }

        [[nodiscard]] bool eof() const noexcept { return eof_; }

        [[nodiscard]] std::vector<Matrix> read_all()
        {
            std::vector<Matrix> all;
            Matrix m;
            while (read_one(m))
                all.push_back(std::move(m));
            return all;
        }

        explicit operator bool() const noexcept { return !eof_; }

    private:
        typename Policy::Reader reader_;
        bool eof_ = false;
    };

    /// Push-style matrix stream over an output policy.
    template <MatrixOutputPolicy Policy>
    class MatrixOutputStream final
    {
    public:
        explicit MatrixOutputStream(const std::filesystem::path &path) : writer_(Policy::open_writer(path)) {}

        void write_one(const Matrix &matrix) { Policy::write_next(writer_, matrix); }

        MatrixOutputStream &operator<<(const Matrix &matrix)
        {
            write_one(matrix);
            return *this;
        }

        void flush() { Policy::flush(writer_); }

        void write_all(std::span<const Matrix> matrices)
        {
            for (const Matrix &m : matrices)
                write_one(m);
            flush();
        }

    private:
        typename Policy::Writer writer_;
    };

    [[nodiscard]] std::vector<Matrix> read_mat_file(const std::filesystem::path &path);
    void write_mat_file(const std::filesystem::path &path, std::span<const Matrix> matrices);
    [[nodiscard]] std::vector<Matrix> read_txt_file(const std::filesystem::path &path);
    void write_txt_file(const std::filesystem::path &path, std::span<const Matrix> matrices);

    using MatInputStream = MatrixInputStream<MatFilePolicy>;
    using MatOutputStream = MatrixOutputStream<MatFilePolicy>;
    using TxtInputStream = MatrixInputStream<TxtFilePolicy>;
    using TxtOutputStream = MatrixOutputStream<TxtFilePolicy>;
} // namespace jacobi::svd::io
