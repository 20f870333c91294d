"""Tile shards: one frame rendered on several GPUs, one process per GPU.

Rank r of n renders the 64x64 film tiles t (numbered row-major) with
t % n == r (sundog_render_ext.shard_count / shard_index); its other pixels
stay 0. A pixel's camera ray and random stream depend only on (pixel,
sample, seed), so every rendered pixel equals the same pixel of a one-GPU
render bit for bit. The one exchange is a gather of the disjoint films at the
end, after which each pixel is taken from the rank that owns its tile
(selection, not a sum: a sum would turn a -0.0 into +0.0).
"""
import numpy as np

TILE = 64


def owner_map(width, height, n):
    """(height, width) int32 array: the rank whose shard holds each pixel."""
    tx = (width + TILE - 1) // TILE
    ty = np.arange(height) // TILE
    tcol = np.arange(width) // TILE
    return ((ty[:, None] * tx + tcol[None, :]) % max(n, 1)).astype(np.int32)


def owned_pixels(width, height, n, rank):
    """Number of film pixels in rank's shard."""
    return int((owner_map(width, height, n) == rank).sum())


def assemble(films):
    """Frame from the n ranks' films (list indexed by rank, each HxWxC)."""
    n = len(films)
    h, w = films[0].shape[:2]
    own = owner_map(w, h, n)
    out = np.zeros_like(films[0])
    for r, f in enumerate(films):
        m = own == r
        out[m] = f[m]
    return out


def session_film(session, device=None):
    """The session's film as a (height, width, 4) float32 torch tensor on the
    session's device (a device-to-device copy on the current stream)."""
    import torch
    st = session.stats
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    film = torch.empty((st.height, st.width, 4), dtype=torch.float32, device=dev)
    session.copy_film(film.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    return film


def gather(film, n, group=None):
    """All-gather of the n ranks' tile-shard films (torch tensors of one shape,
    on the process group's device: CUDA for NCCL, CPU for gloo); returns the
    assembled frame on every rank."""
    import torch
    import torch.distributed as dist
    if n <= 1:
        return film
    parts = [torch.empty_like(film) for _ in range(n)]
    dist.all_gather(parts, film.contiguous(), group=group)
    h, w = film.shape[:2]
    own = torch.from_numpy(owner_map(w, h, n)).to(film.device)
    out = torch.zeros_like(film)
    for r, p in enumerate(parts):
        m = (own == r).unsqueeze(-1)
        out = torch.where(m, p, out)
    return out
