'''CUDA device plumbing shared by the drop-in classes (torch for memory
and streams; the compute is in the C-ABI library).'''
import torch


def get_device(device=None):
    '''The CUDA device to use; RuntimeError without a GPU, as the
    reference's torch backend does (theory/torchLorenzMie.py:178-201).'''
    if not torch.cuda.is_available():
        raise RuntimeError('pylorenzmie_b200 needs a CUDA GPU (sm_100a); '
                           'none is available')
    if device is None:
        return torch.device('cuda', torch.cuda.current_device())
    device = torch.device(device)
    if device.type != 'cuda':
        raise RuntimeError(f'pylorenzmie_b200 runs on CUDA devices, not {device}')
    return device


def stream_handle(device):
    '''cudaStream_t of torch's current stream on device, as an int.'''
    return torch.cuda.current_stream(device).cuda_stream


def ptr(t):
    '''Device address of a tensor (None for None).'''
    return None if t is None else t.data_ptr()
