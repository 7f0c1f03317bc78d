"""CPU stand-in for the two local calls of the multi-GPU build
(distributed_suffix_sorting_evaluation_b200/distributed.py), so that its
exchange steps can run as gloo processes on a machine without a GPU.

TEST INFRASTRUCTURE ONLY: the package has no CPU path; on GPUs the local calls
are the library's radix sort and 32-bit-string build."""
import numpy as np
import torch


class CpuOps:
    device = torch.device("cpu")

    def argsort_words(self, words):
        """Stable lexicographic argsort, words[-1] most significant."""
        if words[0].numel() == 0:
            return torch.zeros(0, dtype=torch.int64)
        return torch.from_numpy(np.lexsort([w.numpy() for w in words]).astype(np.int64))

    def suffix_array(self, s, sigma):
        """Prefix doubling over integer symbols (a different algorithm from the
        one under test; 0 past the end is smaller than every symbol)."""
        a = s.numpy().astype(np.int64)
        n = a.size
        if n == 0:
            return torch.zeros(0, dtype=torch.int64)
        rank = a.copy()
        k = 1
        while True:
            nxt = np.zeros(n, np.int64)
            if k < n:
                nxt[: n - k] = rank[k:]
            order = np.lexsort((nxt, rank))
            r0, r1 = rank[order], nxt[order]
            new = np.empty(n, np.int64)
            new[order] = np.concatenate([[1], 1 + np.cumsum((r0[1:] != r0[:-1]) | (r1[1:] != r1[:-1]))])
            rank = new
            if rank.max() == n:
                return torch.from_numpy(order.astype(np.int64))
            k *= 2
