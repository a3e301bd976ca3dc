"""CPU test of the stream handling of the Python layer
(ncs_b200.ncs.launch_stream), with a fake stream and tensors that report
themselves as CUDA tensors, so that no GPU is needed."""


def test_launch_stream_orders_and_records(monkeypatch):
    """ncs_b200.ncs.launch_stream without a GPU: the current stream is used as
    it is; a caller's other stream first waits for the current one, and the
    CUDA tensors of the launch (not host tensors or None) are recorded on it."""
    import torch
    from ncs_b200 import ncs

    class Stream:
        def __init__(self):
            self.waited = []

        def wait_stream(self, other):
            self.waited.append(other)

    recorded = []

    class FakeCuda(torch.Tensor):
        @property
        def is_cuda(self):
            return True

        def record_stream(self, s):
            recorded.append((id(self), s))

    cur, side = Stream(), Stream()
    monkeypatch.setattr(torch.cuda, "current_stream", lambda device=None: cur)
    a = torch.Tensor._make_subclass(FakeCuda, torch.zeros(2))
    b = torch.Tensor._make_subclass(FakeCuda, torch.zeros(3))
    host = torch.zeros(4)
    # no stream, or the current one: nothing to order or record
    assert ncs.launch_stream(None, "cuda:0", a, host, None) is cur
    assert ncs.launch_stream(cur, "cuda:0", a, host, None) is cur
    assert not recorded and not cur.waited
    # another stream: it waits for the current one; the device tensors are recorded
    assert ncs.launch_stream(side, "cuda:0", a, host, None, b) is side
    assert side.waited == [cur]
    assert recorded == [(id(a), side), (id(b), side)]
