"""HPCsharp's radix-sort extension methods, with the same names, argument meaning and
exceptions, running on the B200 through the C ABI (libhpcs_gpu.so).

Reference surface (paths relative to the HPCsharp project root):
  ParallelAlgorithm.SortRadixPar(this uint[], int ParallelWorkQuantum)  RadixSortLsdParallel.cs:145
  ParallelAlgorithm.SortRadixPar(this int[] / long[] / ulong[])         RadixSortLsdParallel.cs:446, :560, :690
  ParallelAlgorithm.SortRadixInPlaceInterfacePar(this T[])              RadixSortLsdParallel.cs:240, :677, :743
  Algorithm.SortRadixLsd(this T[] [, int start, int length])           RadixSortLsd.cs:255, :352, :437, :527
  Algorithm.SortRadixLsdFunc(this T[] [, int start, int length])       RadixSortLsd.cs:238, :315, :400, :490
  Algorithm.SortRadix(this uint[]) (examples' spelling, Program.cs:26)
  Algorithm.SortRadix<T>(this T[] items, UInt32[]/UInt64[] keys)        RadixSortLsd.cs:1183, :1245
  Algorithm.SortRadixLsd<T>(this T[], Func<T, UInt32/UInt64> getKey)    RadixSortLsd.cs:714, :783
  Algorithm.SortRadixFaster<T>(this T[], Func<T, UInt32/UInt64> getKey) RadixSortLsd.cs:861, :961
  Algorithm.HistogramByteComponents(T[], int l, int r)                 Histogram.cs:261, :957, :992, :1019
  ParallelAlgorithm.HistogramByteComponentsPar(T[], int l, int r, ...)  HistogramParallel.cs:214, :416, :547, :617
  Algorithm.SelectTopK(this uint[], int k) / (a, start, length, k)     SelectionTopKRadix.cs:160, :142
  Algorithm.SortRadixMsd(this float[]/double[]/...)                       RadixSortMsd.cs:1563-1610
  Algorithm.SortCounting[InPlace[Func]](this byte[]/sbyte[]/ushort[]/short[]) CountingSort.cs:23-165
  ParallelAlgorithm.SortCounting[InPlace[Func]]Par(...)                   CountingSortParallel.cs:22-99
  Algorithm.SelectRadix(this uint[]/ulong[], k or int[] k [, start, length])
                                                                       SelectionRadix.cs:236-435
  ParallelAlgorithm.SelectRadixPar(this uint[], [start, length,] k, parallelThreshold)
                                                                       SelectionRadixParallel.cs:254-283
  Algorithm.PartitionRadix(this uint[]/ulong[], [start, length,] k or int[] k, threshold)
                                                                       PartitionRadix.cs:135-210

Arrays are numpy arrays sorted in place (the reference's SortRadixPar returns the caller's
array after an even number of passes, RadixSortLsdParallel.cs:227-231).  float32/float64
keys are accepted too and ordered by the reference's float transform.
"""
from __future__ import annotations

import numpy as np

from .native import (ArgumentNullException, ArgumentOutOfRangeException, HPCS_ERR_NULL, HPCS_ERR_RANGE,
                     default_context)


def _require(a, name: str = "inputArray"):
    if a is None:
        raise ArgumentNullException(HPCS_ERR_NULL, f"{name} is null")


def SortRadixPar(inputArray: np.ndarray, ParallelWorkQuantum: int = 64 * 1024) -> np.ndarray:
    """Stable ascending LSD radix sort, in place; returns the caller's array.  The work
    quantum is the reference's CPU task size and has no effect on the GPU."""
    _require(inputArray)
    return default_context().sort(inputArray)


def SortRadixInPlaceInterfacePar(inputArray: np.ndarray) -> None:
    _require(inputArray)
    default_context().sort(inputArray)


def SortRadixLsd(inOutArray, startIndex=None, length: int | None = None):
    """In-place serial-API sort; with (startIndex, length) sorts that subrange in place.
    (The reference's subrange overload writes its result to [0, length) because
    ComputeStartOfBins starts every bin at 0, RadixSortLsd.cs:120; this sorts the
    subrange where it lies.)

    SortRadixLsd(items, getKey) is the user-defined-type form (RadixSortLsd.cs:714, :783):
    returns a new list of the items in stable ascending order of getKey(item), an unsigned
    32- or 64-bit key (64-bit when any key exceeds 2^32 - 1)."""
    if callable(startIndex):
        return _sort_by_key(inOutArray, startIndex)
    _require(inOutArray, "inOutArray")
    if startIndex is None:
        default_context().sort(inOutArray)
        return
    if length is None or startIndex < 0 or length < 0 or startIndex + length > inOutArray.size:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "startIndex/length outside the array")
    default_context().sort(inOutArray[startIndex:startIndex + length])


def _sort_by_key(inputArray, getKey):
    """Keys extracted on the host, sorted on the GPU with their indices as the payload, items
    gathered by the sorted indices."""
    _require(inputArray, "inputArray")
    _require(getKey, "getKey")
    items = list(inputArray)
    keys = np.fromiter((int(getKey(x)) for x in items), dtype=np.uint64, count=len(items))
    if keys.size and int(keys.max()) <= 0xFFFFFFFF:
        keys = keys.astype(np.uint32)
    index = np.arange(len(items), dtype=np.uint32)
    if len(items):
        default_context().sort_pairs(keys, index)
    return [items[i] for i in index]


def SortRadixFaster(inputArray, getKey):
    """SortRadixFaster<T>(this T[], Func<T, UInt32/UInt64>) RadixSortLsd.cs:861, :961: the
    same stable key-order result as SortRadixLsd(items, getKey)."""
    return _sort_by_key(inputArray, getKey)


def SortRadixLsdFunc(inOutArray: np.ndarray, startIndex: int | None = None, length: int | None = None):
    SortRadixLsd(inOutArray, startIndex, length)
    return inOutArray


def SortRadix(inputArray: np.ndarray, inKeys: np.ndarray | None = None):
    """SortRadix(this uint[]) sorts keys in place and returns them.
    SortRadix<T>(this T[] items, keys) sorts items by keys (stable), permuting both caller
    arrays in place, and returns (items, keys)."""
    if inKeys is None:
        _require(inputArray)
        return default_context().sort(inputArray)
    _require(inputArray)
    _require(inKeys, "inKeys")
    if inputArray.size != inKeys.size:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "items and keys differ in length")
    items = inputArray.view(np.uint32) if inputArray.dtype.itemsize == 4 else None
    if items is None:
        raise TypeError("items must be a 4-byte type (index payload)")
    default_context().sort_pairs(inKeys, items)
    return inputArray, inKeys


def HistogramByteComponentsPar(inArray: np.ndarray, l: int, r: int, parallelThreshold: int = 16 * 1024):
    """uint[P][256] digit counts of inArray[l..r] (inclusive)."""
    _require(inArray, "inArray")
    if l < 0 or r >= inArray.size:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "l/r outside the array")
    return default_context().histogram(inArray, l, r)


def HistogramByteComponents(inArray: np.ndarray, l: int, r: int):
    """int[P][256] digit counts of inArray[l..r] (inclusive)."""
    return HistogramByteComponentsPar(inArray, l, r).astype(np.int32)


def SelectTopK(arrayToBeSelected: np.ndarray, *args) -> None:
    """SelectTopK(a, k) or SelectTopK(a, start, length, k) (SelectionTopKRadix.cs:142-171),
    in place: afterwards a[k] is the k-th smallest and a[k..] the largest of the (sub)array.
    In the (start, length, k) form k indexes the whole array, as in the reference."""
    _require(arrayToBeSelected, "arrayToBeSelected")
    a = arrayToBeSelected
    if len(args) == 1:
        k = args[0]
        if a.size <= 0 or k < 0 or k >= a.size:
            raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "k must be between start and (start + length)")
        default_context().select_topk(a, k)
        return
    start, length, k = args
    if start < 0 or length <= 0 or start + length > a.size:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "l or r are invalid")
    if k < start or k >= start + length:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "k must be between start and (start + length)")
    default_context().select_topk(a[start:start + length], k - start)


def _select_args(a, args, what: str):
    """(start, length, k) from the reference's overloads (k or (start, length, k))."""
    if len(args) == 1:
        if a.size <= 0:
            raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "array length is invalid")
        return 0, a.size, args[0]
    if len(args) == 3:
        start, length, k = args
        if start < 0 or length <= 0 or start + length > a.size:
            raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "array length or length is invalid")
        return int(start), int(length), k
    raise TypeError(f"{what}: expected (k) or (start, length, k)")


def SelectRadix(arrayToBeSelected: np.ndarray, *args):
    """SelectRadix (SelectionRadix.cs:236-435), in place, on the GPU's radix select:
      SelectRadix(a, k) / SelectRadix(a, start, length, k) -> the k-th smallest key of the
        (sub)array (k indexes the whole array), left at a[k] with the (sub)array partitioned
        around it;
      SelectRadix(a, k_list) / SelectRadix(a, start, length, k_list) -> None; afterwards every
        a[k_i] holds the key the sorted (sub)array has at k_i (PartitionRadix by every k)."""
    _require(arrayToBeSelected, "arrayToBeSelected")
    a = arrayToBeSelected
    start, length, k = _select_args(a, args, "SelectRadix")
    if np.ndim(k) == 1:
        PartitionRadix(a, start, length, k)
        return None
    k = int(k)
    if k < start or k >= start + length:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "k must be between start and (start + length)")
    return default_context().select_radix(a, start, length, k)


def SelectRadixPar(arrayToBeSelected: np.ndarray, *args, parallelThreshold: int = 64 * 1024):
    """SelectRadixPar(a, k) / (a, start, length, k) (SelectionRadixParallel.cs:254-283): the k-th
    smallest key of the (sub)array, k indexing the whole array; it is also left at a[k].  The
    parallel threshold is the reference's CPU task size and has no effect on the GPU."""
    _require(arrayToBeSelected, "arrayToBeSelected")
    a = arrayToBeSelected
    start, length, k = _select_args(a, args, "SelectRadixPar")
    k = int(k)
    if k < start or k >= start + length:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "k must be between start and (start + length)")
    return default_context().select_radix(a, start, length, k)


def PartitionRadix(arrayToBePartitioned: np.ndarray, *args, threshold: int = 1024) -> None:
    """PartitionRadix(a, k | k[]) / (a, start, length, k | k[]) (PartitionRadix.cs:135-210), in
    place: afterwards every a[k_i] holds the key the sorted (sub)array has at k_i and the keys
    between two consecutive indices lie between their keys (nth_element).  k indexes the whole
    array.  The base-case threshold is the reference's CPU knob and has no effect on the GPU."""
    _require(arrayToBePartitioned, "arrayToBePartitioned")
    a = arrayToBePartitioned
    start, length, k = _select_args(a, args, "PartitionRadix")
    if k is None:
        raise ArgumentNullException(HPCS_ERR_NULL, "k is null")
    ks = np.atleast_1d(np.asarray(k, dtype=np.int64))
    if ks.size > a.size:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE,
                                          "k array length cannot be greater than the array to be selected length")
    if ks.size == 0:
        return None
    if ((ks < start) | (ks >= start + length)).any():
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "k must be between start and (start + length)")
    default_context().partition_radix(a, start, length, ks)
    return None


def SortRadixMsd(arrayToBeSorted: np.ndarray) -> np.ndarray:
    """SortRadixMsd(this float[]/double[]) RadixSortMsd.cs:1563-1610 (and the integer forms):
    ascending order under the same float/signed transforms, in place.  The LSD sort gives the
    identical result (equal keys are identical bit patterns, so stability is unobservable)."""
    _require(arrayToBeSorted, "arrayToBeSorted")
    return default_context().sort(arrayToBeSorted)


def SortCountingInPlace(arrayToSort: np.ndarray) -> None:
    """SortCountingInPlace(this byte[]/sbyte[]/ushort[]/short[]) CountingSort.cs:41, :78, :115,
    :152: in place, ascending, by the GPU counting sort (one histogram read, one fill)."""
    _require(arrayToSort, "arrayToSort")
    default_context().sort(arrayToSort)


def SortCountingInPlaceFunc(arrayToSort: np.ndarray) -> np.ndarray:
    SortCountingInPlace(arrayToSort)
    return arrayToSort


def SortCounting(inputArray: np.ndarray) -> np.ndarray:
    """SortCounting(this byte[]/...) CountingSort.cs:23: a new sorted array."""
    _require(inputArray, "inputArray")
    out = np.array(inputArray, copy=True)
    default_context().sort(out)
    return out


SortCountingPar = SortCounting
SortCountingInPlacePar = SortCountingInPlace
SortCountingInPlaceFuncPar = SortCountingInPlaceFunc
