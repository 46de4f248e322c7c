// Test driver for include/io.hpp (built and run by tests/test_io.py; no GPU
// needed).  Commands:
//   mat-copy IN OUT        read_mat_file + write_mat_file
//   txt-copy IN OUT        read_txt_file + write_txt_file
//   mat-to-txt IN OUT      MatInputStream -> TxtOutputStream
//   stream-copy IN OUT     MatInputStream >> / MatOutputStream << record by record
//   dispatch IN OUT        MatDispatchReader + decode_dispatch_task_matrix -> *.mat
//                          (needs pinned memory: exits 3 when CUDA is unavailable)
//   dispatch-count IN X    MatDispatchReader over IN, printing the record count
//                          (no device check: for inputs it must refuse before
//                          reserving pinned memory)
// Prints "error: <what>" and exits 1 on an exception.
#include <cuda_runtime.h>

#include <cstring>
#include <exception>
#include <iostream>
#include <string>
#include <vector>

#include "io.hpp"

using namespace jacobi::svd::io;

int main(int argc, char **argv)
{
    if (argc != 4)
        return 64;
    const std::string cmd = argv[1];
    try
    {
        if (cmd == "mat-copy")
        {
            const auto all = read_mat_file(argv[2]);
            write_mat_file(argv[3], all);
        }
        else if (cmd == "txt-copy")
        {
            const auto all = read_txt_file(argv[2]);
            write_txt_file(argv[3], all);
        }
        else if (cmd == "mat-to-txt")
        {
            MatInputStream in(argv[2]);
            TxtOutputStream out(argv[3]);
            Matrix m;
            while (in.read_one(m))
                out << m;
            out.flush();
        }
        else if (cmd == "stream-copy")
        {
            MatInputStream in(argv[2]);
            MatOutputStream out(argv[3]);
            Matrix m;
            std::size_t k = 0;
            while (in >> m, in)
            {
                out << m;
                ++k;
            }
            out.flush();
            std::cout << "records " << k << '\n';
        }
        else if (cmd == "dispatch")
        {
            int count = 0;
            if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
                return 3;
            MatDispatchReader reader(argv[2]);
            MatDispatchTask task;
            std::vector<Matrix> out;
            while (reader.read_next(task, 128))
            {
                if (task.sequence_index != out.size() || task.buffer.workspace_size_bytes() != 128)
                    throw std::runtime_error("dispatch bookkeeping mismatch");
                out.push_back(decode_dispatch_task_matrix(task));
            }
            write_mat_file(argv[3], out);
        }
        else if (cmd == "dispatch-count")
        {
            MatDispatchReader reader(argv[2]);
            MatDispatchTask task;
            std::size_t k = 0;
            while (reader.read_next(task, 0))
                ++k;
            std::cout << "records " << k << '\n';
        }
        else
        {
            return 64;
        }
    }
    catch (const std::exception &e)
    {
        std::cout << "error: " << e.what() << '\n';
        return 1;
    }
    return 0;
}
